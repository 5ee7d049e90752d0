// The low-|k| set of the mixed path on the tensor cores, in 32-bit fixed point.
//
// The k-vectors with |k| < ksplit alpha carry most of the error weight of the
// reciprocal sum (A_k |k| peaks near alpha), so the 24-bit kernels of
// ewald_tc.cuh leave them out.  Here the same factorised GEMMs run on them
// with every operand value a 32-bit fixed-point integer in four signed int8
// digits: the ten digit products of weight >= 2^24 (of 2^48 for the leading
// pair) accumulate exactly in four S32 levels of tensor memory, and the
// operands are generated from FP64 tables, so the error is the 32-bit
// quantisation (2.3e-10 of the scale per term) instead of 6e-8.
//
//   structure factor  S[c, nz] = sum_a A0[c,a] Z_a[nz] + A1[c,a] (i nz/kz) Z_a[nz]
//                     (rows = low-set columns (nx, ny), N = (nz, re/im));
//   field             F_j[i, c] = sum_nz Z_i[nz] nz^j conj(a[c, nz])
//                     (rows = 128-atom tiles, N = (column, moment, re/im)),
// the same decompositions as ewald_tc.cuh.  The nz = 0 row (Z = 1) stays out
// of both GEMMs, so the 2 kz rows nz = -kz..-1, 1..kz fill K = 32 bytes (N =
// 32) up to kz = 8: S[c, 0] = sum_a A0[c, a] is summed in FP64 by the
// producers, and conj(a[c, 0]) enters the field epilogue as a per-column
// constant.  The structure factor writes the
// per-split partials of the FP64 low-set kernels (k_sfac64_low_reduce forms
// A_k S(k), energy and stress), the field pass the low set's field parts
// (k_kfield_reduce adds them).  All column-dependent sums of the field
// epilogue are FP64.
#pragma once
#include "umma.cuh"

namespace mdff {
namespace tc4 {

constexpr int ND = 4;                  // int8 digits per value
constexpr int SA = 16;                 // atoms per pipeline stage
constexpr int KB = 4 * SA;             // K bytes per operand row per stage
constexpr int MAXIN = 8;               // deepest input pipeline
constexpr int NA = 4;                  // A-operand buffers
constexpr int NPW = 16;                // producer warps
constexpr int THREADS = 32 * (NPW + 2);   // + MMA warp + copy warp
constexpr int LS = 64;                 // N <= LS: the four levels of N columns fit ND * LS
constexpr int A_SLICE = 128 * KB;
constexpr int MAX_ATOMS_PER_CTA = 8192;   // S32 headroom: 4 products of 2^14 per K byte at the lowest level
constexpr uint64_t WAIT_NS = 200000000ull;

// Shared memory: NA A-operand buffers (the producers' digit images), then
// nin input buffers (a stage's B digit image, X/Y tables and parameters),
// so the copies run up to nin stages ahead of the producers.
struct Layout {
    int N, XYW, nin;
    uint32_t a_bytes, in_off, b_off, xy_off, p_off, in_bytes;
    __host__ __device__ static uint32_t up128(uint32_t x) { return (x + 127u) & ~127u; }
    __host__ __device__ Layout(int N_, int XYW_, int nin_) : N(N_), XYW(XYW_), nin(nin_) {
        a_bytes = (uint32_t)ND * A_SLICE;
        in_off = NA * a_bytes;
        b_off = 0;
        xy_off = up128((uint32_t)ND * N * KB);
        p_off = up128(xy_off + (uint32_t)SA * XYW * 16u);
        in_bytes = up128(p_off + (uint32_t)SA * 32u);
    }
    __host__ __device__ uint32_t b_bytes() const { return (uint32_t)ND * N * KB; }
    __host__ __device__ uint32_t smem_bytes() const { return in_off + (uint32_t)nin * in_bytes + 128u; }
    // the deepest input pipeline (<= MAXIN) that fits in `limit` bytes, 0 if none of 2 does
    __host__ static int depth(int N_, int XYW_, size_t limit) {
        for (int d = MAXIN; d >= 2; --d)
            if (Layout(N_, XYW_, d).smem_bytes() <= limit) return d;
        return 0;
    }
};

// nz of GEMM row m (rows nz = -kz..-1, then 1..kz)
__host__ __device__ __forceinline__ int row_nz(int m, int kz) { return m < kz ? m - kz : m - kz + 1; }

__device__ __forceinline__ void phase64(uint32_t ph, double& c, double& s) {
    sincospi((double)(int)ph * 4.656612873077393e-10, &s, &c);   // 2 pi t, t = ph / 2^32
}

// Per position update: X_a[nx] (nx = 0..kx) then Y_a[ny] (ny = -ky..ky) per
// atom in FP64, padded to XYW entries; atoms past n get (1, 0).
__global__ void k_tc4_xy(int n, int npad, const uint32_t* __restrict__ fx, int kx, int ky, int XYW,
                         double2* __restrict__ xy) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)npad * XYW) return;
    const int a = (int)(t / XYW), e = (int)(t % XYW);
    double2 v = make_double2(0.0, 0.0);
    if (a >= n) {
        v = make_double2(1.0, 0.0);
    } else if (e <= kx) {
        phase64((uint32_t)e * fx[a], v.x, v.y);
    } else if (e <= kx + 1 + 2 * ky) {
        const int ny = e - (kx + 1) - ky;
        phase64((uint32_t)ny * fx[n + a], v.x, v.y);
    }
    xy[t] = v;
}

// Per position update: the structure factor's B digit image (rows 2m, 2m+1 =
// re, im of GEMM row m, nz = row_nz(m); the four K entries of each atom), one
// thread per (atom, row m), in the K-major core-matrix layout of one stage.
__global__ void k_tc4_bimage(int n, int npad, const uint32_t* __restrict__ fx, int kz, int nzl, int N,
                             uint8_t* __restrict__ img) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int half = N / 2;
    if (t >= (long)npad * half) return;
    const int a = (int)(t / half), m = (int)(t % half);
    double b[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (a < n && m < nzl) {
        const int nz = row_nz(m, kz);
        double zc, zs;
        phase64((uint32_t)nz * fx[2 * n + a], zc, zs);
        const double f = kz > 0 ? (double)nz / (double)kz : 0.0;
        const double b1r = -f * zs, b1i = f * zc;     // i (nz/kz) Z
        b[0] = zc;  b[1] = -zs; b[2] = b1r; b[3] = -b1i;
        b[4] = zs;  b[5] = zc;  b[6] = b1i; b[7] = b1r;
    }
    // the four digit slices side by side along N (rows d N + r), so that one
    // MMA multiplies an A slice by all the B slices it pairs with
    const int blk = a / SA, al = a % SA;
    uint8_t* base = img + (size_t)blk * ND * N * KB;
    const uint32_t lbo = (uint32_t)(ND * N / 8) * 128, sstep = (uint32_t)(N / 8) * 128;
#pragma unroll
    for (int row = 0; row < 2; ++row) {
        const int r = 2 * m + row;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = umma::digits32(__double2int_rn(b[4 * row + j] * umma::QS4));
        uint32_t s[ND];
        umma::slices4x4(w[0], w[1], w[2], w[3], s[0], s[1], s[2], s[3]);
        const uint32_t off = (uint32_t)(al >> 2) * lbo + (uint32_t)(r >> 3) * 128 + (r & 7) * 16 + 4 * (al & 3);
#pragma unroll
        for (int d = 0; d < ND; ++d) *reinterpret_cast<uint32_t*>(base + (uint32_t)d * sstep + off) = s[d];
    }
}

// Per evaluation: (q, m1, m2, m3) per atom in FP64 and the bound
// max(|q| + kx |m1| + ky |m2|, kz |m3|) of the amplitudes.
__global__ void k_tc4_params(int n, int npad, const double* __restrict__ q, const double* __restrict__ mu, CellP c,
                             int with_q, int with_mu, int kx, int ky, int kz, double4* __restrict__ prm,
                             double* __restrict__ amax) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= npad) return;
    double qa = 0, m1 = 0, m2 = 0, m3 = 0;
    if (a < n) {
        if (with_q) qa = q[a];
        if (with_mu) {
            const double u0 = mu[a], u1 = mu[n + a], u2 = mu[2 * n + a];
            m1 = 2.0 * PI * (c.B[0] * u0 + c.B[3] * u1 + c.B[6] * u2);
            m2 = 2.0 * PI * (c.B[1] * u0 + c.B[4] * u1 + c.B[7] * u2);
            m3 = 2.0 * PI * (c.B[2] * u0 + c.B[5] * u1 + c.B[8] * u2);
        }
    }
    prm[a] = make_double4(qa, m1, m2, m3);
    amax[a] = fmax(fabs(qa) + kx * fabs(m1) + ky * fabs(m2), kz * fabs(m3));
}

__device__ __forceinline__ bool tc_wait(uint64_t* b, uint32_t parity, int* err, int code, volatile int* stop) {
    if (umma::mbar_wait_ns(b, parity, WAIT_NS, stop)) return true;
    if (!*stop) atomicOr(err, code);
    *stop = 1;
    return false;
}

// Structure factor of the low set.  grid (tiles of 128 list columns, atom
// splits); THREADS threads; dynamic shared memory Layout::smem_bytes().
// cols: the low list [ncol][4] = nx, ny, nzlo, nzn.  Writes
// part[split][mz][column] for mz < nzmax (zero past the column's nzn).
__global__ void __launch_bounds__(THREADS, 1)
    k_sfac_tc4(int nblk, int bps, int nin, const uint8_t* __restrict__ bimg, const double2* __restrict__ xy,
               const double4* __restrict__ prm, const double* __restrict__ amax, const int* __restrict__ cols,
               int ncol, int nzmax, int kx, int ky, int kz, int N, int XYW, double* __restrict__ part_re,
               double* __restrict__ part_im, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t infull[MAXIN], inempty[MAXIN], afull[NA], aempty[NA], done;
    __shared__ uint32_t tslot;
    __shared__ double red[THREADS / 32];
    __shared__ double2 zsum[4][128];   // per producer group h: sum of A0 over its atoms (the nz = 0 row)
    __shared__ volatile int stop;
    const Layout L(N, XYW, nin);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x, split = blockIdx.y;
    const int blk0 = split * bps, blk1 = min(nblk, blk0 + bps);
    const int nst = max(0, blk1 - blk0);

    double mx = 0.0;
    for (int a = blk0 * SA + tid; a < blk1 * SA; a += THREADS) mx = fmax(mx, amax[a]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    if (tid == 0) {
        for (int b = 0; b < nin; ++b) {
            umma::mbar_init(&infull[b], 1);
            umma::mbar_init(&inempty[b], 1);
        }
        for (int b = 0; b < NA; ++b) {
            umma::mbar_init(&afull[b], NPW);
            umma::mbar_init(&aempty[b], 1);
        }
        umma::mbar_init(&done, 1);
        stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) umma::tmem_alloc(&tslot, ND * LS);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    double sigma = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) sigma = fmax(sigma, red[w]);
    // a CTA whose amplitudes all vanish (e.g. a solver direction zero on its
    // atoms) contributes exact zeros; QS4 / sigma must stay finite
    const double inv = sigma > 1e-280 ? umma::QS4 / sigma : 0.0;
    const uint32_t sbase = umma::smem_u32(smem);

    if (warp < NPW) {
        // ---- producers: row r of the A tile, atoms [4h, 4h + 4) of each stage
        const int r = tid & 127, h = tid >> 7;
        const int li = tile * 128 + r;
        const bool valid = li < ncol;
        const int nx = valid ? cols[4 * li] : 0, ny = valid ? cols[4 * li + 1] : 0;
        const double rinv = valid ? inv : 0.0;
        const double fnx = (double)nx * rinv, fny = (double)ny * rinv, gk = (double)kz * rinv;
        const int ex = nx, ey = kx + 1 + ny + ky;
        const uint32_t off = (uint32_t)h * (16 * 128) + (uint32_t)(r >> 3) * 128 + (r & 7) * 16;
        double z0r = 0.0, z0i = 0.0;
        for (int s = 0; s < nst; ++s) {
            const int bi = s % nin, ba = s % NA;
            if (!tc_wait(&infull[bi], (s / nin) & 1, err, 2, &stop)) break;
            if (s >= NA && !tc_wait(&aempty[ba], ((s / NA) - 1) & 1, err, 32, &stop)) break;
            const uint8_t* ib = smem + L.in_off + bi * L.in_bytes;
            const double2* sxy = reinterpret_cast<const double2*>(ib + L.xy_off);
            const double4* sp = reinterpret_cast<const double4*>(ib + L.p_off);
            uint32_t w[ND][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int al = 4 * h + u;
                const double2 X = sxy[al * XYW + ex], Y = sxy[al * XYW + ey];
                const double4 P = sp[al];
                const double xr = fma(X.x, Y.x, -X.y * Y.y), xi = fma(X.x, Y.y, X.y * Y.x);
                const double ar = P.x * rinv, ai = fma(fnx, P.y, fny * P.z), gg = P.w * gk;
                const double a0r = fma(xr, ar, -xi * ai), a0i = fma(xr, ai, xi * ar);
                const double a1r = xr * gg, a1i = xi * gg;
                z0r += a0r;
                z0i += a0i;
                umma::slices4x4(umma::digits32(umma::rint_i32(a0r)), umma::digits32(umma::rint_i32(a0i)),
                                umma::digits32(umma::rint_i32(a1r)), umma::digits32(umma::rint_i32(a1i)), w[0][u],
                                w[1][u], w[2][u], w[3][u]);
            }
            uint8_t* ab = smem + ba * L.a_bytes;
#pragma unroll
            for (int d = 0; d < ND; ++d)
                *reinterpret_cast<uint4*>(ab + d * A_SLICE + off) = make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
            umma::fence_smem_to_async();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&afull[ba]);
        }
        zsum[h][r] = make_double2(z0r, z0i);
        asm volatile("bar.sync 1, %0;" ::"r"(NPW * 32) : "memory");   // the producers only
    } else if (warp == NPW + 1) {
        // ---- copies: B digit image, X/Y tables and parameters of each stage,
        // up to nin stages ahead
        if (lane == 0) {
            const uint32_t bytes = L.b_bytes() + SA * XYW * 16u + SA * 32u;
            int last = -1;
            for (int s = 0; s < nst; ++s) {
                const int bi = s % nin, blk = blk0 + s;
                if (s >= nin && !tc_wait(&inempty[bi], ((s / nin) - 1) & 1, err, 1, &stop)) break;
                uint8_t* ib = smem + L.in_off + bi * L.in_bytes;
                umma::mbar_arrive_expect_tx(&infull[bi], bytes);
                umma::bulk_g2s(ib + L.b_off, bimg + (size_t)blk * L.b_bytes(), L.b_bytes(), &infull[bi]);
                umma::bulk_g2s(ib + L.xy_off, xy + (size_t)blk * SA * XYW, SA * XYW * 16u, &infull[bi]);
                umma::bulk_g2s(ib + L.p_off, prm + (size_t)blk * SA, SA * 32u, &infull[bi]);
                last = s;
            }
            // every copy issued has landed before the CTA can exit, also when the
            // pipeline was abandoned on an error (bounded, whatever the stop flag)
            for (int k = max(0, last - nin + 1); k <= last; ++k) umma::mbar_wait_ns(&infull[k % nin], (k / nin) & 1, WAIT_NS);
        }
    } else if (lane == 0) {
        // ---- MMA issue: per stage 2 K-steps of 32 x the ten digit products as
        // four MMAs: A digit i times B digits 0..3-i (side by side along N,
        // width (4-i) N <= 256) into levels i..3, which sit N columns apart
        uint32_t idesc[ND];
#pragma unroll
        for (int i = 0; i < ND; ++i) idesc[i] = umma::idesc_s8(128, (ND - i) * N);
        const uint32_t lboA = 16 * 128, lboB = (uint32_t)(ND * N / 8) * 128;
        const uint64_t adesc0 = umma::desc_kmajor(sbase, lboA, 128);
        const uint64_t bdesc0 = umma::desc_kmajor(sbase + L.in_off + L.b_off, lboB, 128);
        const uint32_t astep = L.a_bytes >> 4, instep = L.in_bytes >> 4;
        const uint32_t aslice = A_SLICE >> 4;
        for (int s = 0; s < nst; ++s) {
            const int bi = s % nin, ba = s % NA;
            if (!tc_wait(&infull[bi], (s / nin) & 1, err, 4, &stop)) break;
            if (!tc_wait(&afull[ba], (s / NA) & 1, err, 8, &stop)) break;
            umma::fence_after_sync();
            const uint64_t ab = adesc0 + (uint64_t)(ba * astep), bb = bdesc0 + (uint64_t)(bi * instep);
#pragma unroll
            for (int ks = 0; ks < KB / 32; ++ks)
#pragma unroll
                for (int i = 0; i < ND; ++i) {
                    const uint64_t ad = ab + (uint64_t)(i * aslice + ((2 * ks * lboA) >> 4));
                    const uint64_t bd = bb + (uint64_t)((2 * ks * lboB) >> 4);
                    const uint32_t acc = (s > 0 || ks > 0 || i > 0) ? 1u : 0u;
                    umma::mma_s8(tmem + (uint32_t)(i * N), ad, bd, idesc[i], acc);
                }
            umma::commit(&inempty[bi]);
            umma::commit(&aempty[ba]);
        }
        umma::commit(&done);
    }

    // ---- epilogue: warps 0-3 (tensor-memory lane quarters), row = thread
    if (warp < 4) {
        const bool ok = nst == 0 || tc_wait(&done, 0, err, 16, &stop);
        umma::fence_after_sync();
        const int li = tile * 128 + tid;
        const bool valid = li < ncol;
        const int nzlo = valid ? cols[4 * li + 2] : 0, nzn = valid ? cols[4 * li + 3] : 0;
        const size_t plane = (size_t)nzmax * ncol, base = (size_t)split * plane + li;
        if (valid)
            for (int mz = nzn; mz < nzmax; ++mz) {
                part_re[base + (size_t)mz * ncol] = 0.0;
                part_im[base + (size_t)mz * ncol] = 0.0;
            }
        const double osc = sigma / (umma::QS4 * umma::QS4);
        const int mz0 = -nzlo;   // the nz = 0 row, summed by the producers
        if (valid && ok && mz0 >= 0 && mz0 < nzn) {
            const double sc = sigma / umma::QS4;
            double zr = 0.0, zi = 0.0;
            for (int hh = 0; hh < 4; ++hh) { zr += zsum[hh][tid].x; zi += zsum[hh][tid].y; }
            part_re[base + (size_t)mz0 * ncol] = zr * sc;
            part_im[base + (size_t)mz0 * ncol] = zi * sc;
        }
        const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
        for (int j = 0; j < N / 16; ++j) {
            float d[ND][16];
            if (nst > 0) {
#pragma unroll
                for (int l = 0; l < ND; ++l) umma::tmem_ld16(lane_base + l * N + 16 * j, d[l]);
                umma::tmem_wait_ld();
            }
            if (!valid || !ok) continue;
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int nn = 16 * j + e;
                const int mz = row_nz(nn >> 1, kz) - nzlo;
                if (mz < 0 || mz >= nzn) continue;
                double v = 0.0;
                if (nst > 0)
                    v = ((double)__float_as_int(d[0][e]) * 281474976710656.0 +
                         (double)__float_as_int(d[1][e]) * 1099511627776.0 +
                         (double)__float_as_int(d[2][e]) * 4294967296.0 + (double)__float_as_int(d[3][e]) * 16777216.0) *
                        osc;
                if (nn & 1) part_im[base + (size_t)mz * ncol] = v;
                else part_re[base + (size_t)mz * ncol] = v;
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, ND * LS);
    }
}

// ===========================================================================
// Field pass of the low set.  M = 128 atoms per CTA, K = (nz row, re/im) of
// Z_i[nz], N = (column, moment, re/im) in blocks of CB columns; the
// contraction over columns runs in FP64 in the epilogue (16 warps: each
// atom's row split over four warps by column quarters), double-buffered in
// tensor memory against the next block's MMAs.

constexpr int EPW = 16;                  // epilogue warps: 4 per tensor-memory lane quarter
constexpr int NQ = EPW / 4;
constexpr int FTHREADS = 32 * (EPW + 2);
constexpr int NBS = 4;                   // B stages
constexpr int TMEM_COLS = 512;           // two accumulator buffers of ND levels of NB columns
constexpr int NCONST = 16;               // doubles of per-column constants

template <int NMOM>
struct Cfg {
    static constexpr int CB = NMOM == 2 ? 16 : 8;   // columns per block
    static constexpr int NB = CB * NMOM * 2;        // GEMM N per block (64 or 48)
    static constexpr int HC = CB / NQ;              // columns per epilogue warp
    static constexpr int WN = HC * NMOM * 2;        // accumulator columns per warp per level (16 or 12)
    static constexpr int BUFC = ND * NB;            // per accumulator buffer (levels NB columns apart)
    static_assert(2 * BUFC <= TMEM_COLS, "two accumulator buffers");
};

struct FLayout {
    int KZ, XYW, NB, CB;
    uint32_t a_off, xy_off, b_off, stage_bytes, img_bytes;
    __host__ __device__ static uint32_t up128(uint32_t x) { return (x + 127u) & ~127u; }
    __host__ __device__ FLayout(int KZ_, int XYW_, int NB_, int CB_) : KZ(KZ_), XYW(XYW_), NB(NB_), CB(CB_) {
        a_off = 0;
        xy_off = up128((uint32_t)ND * 128u * KZ);
        b_off = up128(xy_off + (uint32_t)XYW * 128u * 16u);
        img_bytes = (uint32_t)ND * NB * KZ + (uint32_t)CB * NCONST * 8u;
        stage_bytes = up128(img_bytes);
    }
    __host__ __device__ uint32_t a_bytes() const { return (uint32_t)ND * 128u * KZ; }
    __host__ __device__ uint32_t xy_bytes() const { return (uint32_t)XYW * 128u * 16u; }
    __host__ __device__ uint32_t smem_bytes() const { return b_off + NBS * stage_bytes + 128u; }
};

// Per position update: the A digit image of each 128-atom tile (rows = atoms,
// K = (GEMM row m, re/im) of Z_i[row_nz(m)]; KZ bytes per row, zero past 2 nzl).
__global__ void k_tc4f_aimage(int n, int ntile, const uint32_t* __restrict__ fx, int kz, int nzl, int KZ,
                              uint8_t* __restrict__ img) {
    const int nch = KZ / 16;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ntile * 128 * nch) return;
    const int kc = (int)(t % nch);
    const int a = (int)(t / nch);
    const int tile = a / 128, r = a % 128;
    double v[16];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int m = 8 * kc + u;
        double zc = 0.0, zs = 0.0;
        if (a < n && m < nzl) phase64((uint32_t)row_nz(m, kz) * fx[2 * n + a], zc, zs);
        v[2 * u] = zc * umma::QS4;
        v[2 * u + 1] = zs * umma::QS4;
    }
    uint32_t s[ND][4];
#pragma unroll
    for (int g = 0; g < 4; ++g)
        umma::slices4x4(umma::digits32(__double2int_rn(v[4 * g])), umma::digits32(__double2int_rn(v[4 * g + 1])),
                        umma::digits32(__double2int_rn(v[4 * g + 2])), umma::digits32(__double2int_rn(v[4 * g + 3])),
                        s[0][g], s[1][g], s[2][g], s[3][g]);
    uint8_t* base = img + (size_t)tile * ND * 128 * KZ;
    const uint32_t off = (uint32_t)kc * (16 * 128) + (uint32_t)(r >> 3) * 128 + (r & 7) * 16;
#pragma unroll
    for (int d = 0; d < ND; ++d)
        *reinterpret_cast<uint4*>(base + (size_t)d * 128 * KZ + off) = make_uint4(s[d][0], s[d][1], s[d][2], s[d][3]);
}

// Per position update: the FP64 X/Y tables of each tile transposed to [tile][entry][128].
__global__ void k_tc4f_xyt(int npad, int ntile, const double2* __restrict__ xy, int XYW, double2* __restrict__ xyt) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ntile * 128 * XYW) return;
    const int r = (int)(t % 128);
    const long te = t / 128;
    const int e = (int)(te % XYW), tile = (int)(te / XYW);
    const int a = tile * 128 + r;
    xyt[t] = a < npad ? xy[(size_t)a * XYW + e] : make_double2(0.0, 0.0);
}

// Per evaluation: the B digit image and per-column constants of each column
// block of the low list.  Block = one column block, thread = (GEMM row n,
// 16-byte K chunk).  aks: the low set's A_k S(k), [2][ncol][nzmax].
// Constants per column (FP64): s0, s1, s2, kc (3), kc_d kc_e (00 11 22 01 02
// 12), conj(a[c, 0]) (2), X entry, Y entry; s_j = (scale of moment j) 2^24 /
// QS4^2.
template <int NMOM>
__global__ void k_tc4f_bimage(int ncol, const int* __restrict__ cols, int nzmax, int kx, int ky, int kz, int nzl,
                              int KZ, const double* __restrict__ aks, CellP c, uint8_t* __restrict__ img) {
    using C = Cfg<NMOM>;
    const int nch = KZ / 16;
    const FLayout L(KZ, 0, C::NB, C::CB);
    __shared__ unsigned long long smax[C::CB * NMOM];
    const int q = blockIdx.x, t = threadIdx.x;
    if (t < C::CB * NMOM) smax[t] = 0ull;
    __syncthreads();
    const int n = t / nch, kc = t % nch;
    const int cl = n / (2 * NMOM), j = (n >> 1) % NMOM, part = n & 1;
    const int li = q * C::CB + cl;
    const bool valid = li < ncol;
    const int nzlo = valid ? cols[4 * li + 2] : 0, nzn = valid ? cols[4 * li + 3] : 0;
    double br[8], bi[8];   // nz^j conj(a) over the chunk's 8 rows
    double mx = 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int m = 8 * kc + u;
        const int nz = row_nz(m, kz), mz = nz - nzlo;
        br[u] = 0.0; bi[u] = 0.0;
        if (valid && m < nzl && mz >= 0 && mz < nzn) {
            const double w = j == 0 ? 1.0 : (j == 1 ? (double)nz : (double)nz * (double)nz);
            const size_t r = (size_t)li * nzmax + mz;
            br[u] = w * aks[r];
            bi[u] = -w * aks[(size_t)ncol * nzmax + r];
        }
        mx = fmax(mx, fmax(fabs(br[u]), fabs(bi[u])));
    }
    if (t < nch * C::NB) atomicMax(&smax[cl * NMOM + j], (unsigned long long)__double_as_longlong(mx));
    __syncthreads();
    uint8_t* base = img + (size_t)q * L.stage_bytes;
    if (t < nch * C::NB) {
        const double sg = __longlong_as_double((long long)smax[cl * NMOM + j]);
        const double qsc = sg > 1e-280 ? umma::QS4 / sg : 0.0;
        double v[16];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            // part re: (Re B, -Im B); part im: (Im B, Re B)
            v[2 * u] = (part ? bi[u] : br[u]) * qsc;
            v[2 * u + 1] = (part ? br[u] : -bi[u]) * qsc;
        }
        uint32_t s[ND][4];
#pragma unroll
        for (int g = 0; g < 4; ++g)
            umma::slices4x4(umma::digits32(__double2int_rn(v[4 * g])), umma::digits32(__double2int_rn(v[4 * g + 1])),
                            umma::digits32(__double2int_rn(v[4 * g + 2])),
                            umma::digits32(__double2int_rn(v[4 * g + 3])), s[0][g], s[1][g], s[2][g], s[3][g]);
        // the four digit slices side by side along N (rows d NB + n)
        const uint32_t lbo = (uint32_t)(ND * C::NB / 8) * 128, sstep = (uint32_t)(C::NB / 8) * 128;
        const uint32_t off = (uint32_t)kc * lbo + (uint32_t)(n >> 3) * 128 + (n & 7) * 16;
#pragma unroll
        for (int d = 0; d < ND; ++d)
            *reinterpret_cast<uint4*>(base + d * sstep + off) = make_uint4(s[d][0], s[d][1], s[d][2], s[d][3]);
    }
    if (t < C::CB) {
        double* k = reinterpret_cast<double*>(base + (size_t)ND * C::NB * KZ) + t * NCONST;
        const int li2 = q * C::CB + t;
        double cv[NCONST];
#pragma unroll
        for (int e = 0; e < NCONST; ++e) cv[e] = 0.0;
        if (li2 < ncol) {
            const int nx = cols[4 * li2], ny = cols[4 * li2 + 1];
            const double w = 16777216.0 / (umma::QS4 * umma::QS4);
            for (int jj = 0; jj < 3; ++jj)
                cv[jj] = jj < NMOM ? __longlong_as_double((long long)smax[t * NMOM + jj]) * w : 0.0;
            double kc3[3];
            for (int d = 0; d < 3; ++d) kc3[d] = 2.0 * PI * (nx * c.B[3 * d] + ny * c.B[3 * d + 1]);
            cv[3] = kc3[0]; cv[4] = kc3[1]; cv[5] = kc3[2];
            cv[6] = kc3[0] * kc3[0]; cv[7] = kc3[1] * kc3[1]; cv[8] = kc3[2] * kc3[2];
            cv[9] = kc3[0] * kc3[1]; cv[10] = kc3[0] * kc3[2]; cv[11] = kc3[1] * kc3[2];
            const int mz0 = -cols[4 * li2 + 2];
            if (mz0 >= 0 && mz0 < cols[4 * li2 + 3]) {
                cv[12] = aks[(size_t)li2 * nzmax + mz0];
                cv[13] = -aks[(size_t)ncol * nzmax + (size_t)li2 * nzmax + mz0];
            }
            cv[14] = (double)nx;
            cv[15] = (double)(kx + 1 + ny + ky);
        }
#pragma unroll
        for (int e = 0; e < NCONST; ++e) k[e] = cv[e];
    }
}

// exact digit-level sums -> FP64: (D0 2^8 + D1) 2^16 + (D2 2^8 + D3), an
// integer below 2^51 (each half stays inside int32 for K <= 128 bytes),
// converted on the FP64 pipe; the common 2^24 and the column scale live in
// the per-column constants.
__device__ __forceinline__ double comb4(float d0, float d1, float d2, float d3) {
    const int hi = __float_as_int(d0) * 256 + __float_as_int(d1);
    const int lo = __float_as_int(d2) * 256 + __float_as_int(d3);
    return umma::i64_to_f64((long long)hi * 65536ll + (long long)lo);
}

// grid = 128-atom tiles; FTHREADS threads; dynamic shared memory FLayout::smem_bytes().
// Writes fpart[(part * 9 + component) * n + i] for the NQ column parts
// (components 0-2 the field, 3-8 the field gradient when NMOM = 3).
template <int NMOM>
__global__ void __launch_bounds__(FTHREADS, 1)
    k_kfield_tc4(int n, int ncb, const uint8_t* __restrict__ aimg, const double2* __restrict__ xyt,
                 const uint8_t* __restrict__ bimg, int KZ, int XYW, CellP c, double* __restrict__ fpart,
                 int* __restrict__ err) {
    using C = Cfg<NMOM>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t ares, bfull[NBS], bempty[NBS], accfull[2], accfree[2], fin;
    __shared__ uint32_t tslot;
    __shared__ volatile int abort_;
    const FLayout L(KZ, XYW, C::NB, C::CB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x;
    if (tid == 0) {
        umma::mbar_init(&ares, 1);
        for (int b = 0; b < NBS; ++b) {
            umma::mbar_init(&bfull[b], 1);
            umma::mbar_init(&bempty[b], 1 + EPW);
        }
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(&accfull[b], 1);
            umma::mbar_init(&accfree[b], EPW);
        }
        umma::mbar_init(&fin, 1);
        abort_ = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) umma::tmem_alloc(&tslot, TMEM_COLS);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t sbase = umma::smem_u32(smem);

    if (warp == EPW + 1) {
        // ---- copies: the tile's A image and X/Y table, then the B stages
        if (lane == 0) {
            umma::mbar_arrive_expect_tx(&ares, L.a_bytes() + L.xy_bytes());
            umma::bulk_g2s(smem + L.a_off, aimg + (size_t)tile * L.a_bytes(), L.a_bytes(), &ares);
            umma::bulk_g2s(smem + L.xy_off, xyt + (size_t)tile * XYW * 128, L.xy_bytes(), &ares);
            int last = -1;
            for (int q = 0; q < ncb; ++q) {
                const int bs = q % NBS;
                if (q >= NBS && !tc_wait(&bempty[bs], ((q / NBS) - 1) & 1, err, 1, &abort_)) break;
                umma::mbar_arrive_expect_tx(&bfull[bs], L.img_bytes);
                umma::bulk_g2s(smem + L.b_off + bs * L.stage_bytes, bimg + (size_t)q * L.stage_bytes, L.img_bytes,
                               &bfull[bs]);
                last = q;
            }
            // every copy issued has landed before the CTA can exit, also when the
            // pipeline was abandoned on an error (bounded, whatever the stop flag)
            umma::mbar_wait_ns(&ares, 0, WAIT_NS);
            for (int k = max(0, last - NBS + 1); k <= last; ++k) umma::mbar_wait_ns(&bfull[k % NBS], (k / NBS) & 1, WAIT_NS);
        }
    } else if (warp == EPW) {
        // ---- MMA issue (the whole warp, one elected lane issues): per column
        // block KZ/32 K-steps x 4 MMAs, A digit i times B digits 0..3-i (side
        // by side along N) into levels i..3: the ten digit products, each A
        // slice read once per K-step
        {
            uint32_t idesc[ND];
#pragma unroll
            for (int i = 0; i < ND; ++i) idesc[i] = umma::idesc_s8(128, (ND - i) * C::NB);
            const uint32_t lboA = 16 * 128, lboB = (uint32_t)(ND * C::NB / 8) * 128;
            const uint64_t adesc0 = umma::desc_kmajor(sbase + L.a_off, lboA, 128);
            const uint64_t bdesc0 = umma::desc_kmajor(sbase + L.b_off, lboB, 128);
            const uint32_t aslice = (128u * KZ) >> 4;
            const uint32_t astep = (2 * lboA) >> 4, bkstep = (2 * lboB) >> 4, bstage = L.stage_bytes >> 4;
            bool ok = __all_sync(0xffffffffu, tc_wait(&ares, 0, err, 2, &abort_));
            for (int q = 0; q < ncb && ok; ++q) {
                const int bs = q % NBS, tb = q & 1;
                ok = __all_sync(0xffffffffu, tc_wait(&bfull[bs], (q / NBS) & 1, err, 4, &abort_));
                if (ok && q >= 2) ok = __all_sync(0xffffffffu, tc_wait(&accfree[tb], ((q >> 1) - 1) & 1, err, 8, &abort_));
                if (!ok) break;
                umma::fence_after_sync();
                const uint64_t bq = bdesc0 + (uint64_t)(bs * bstage);
                for (int ks = 0; ks < KZ / 32; ++ks) {
#pragma unroll
                    for (int i = 0; i < ND; ++i) {
                        const uint64_t ad = adesc0 + (uint64_t)(i * aslice + ks * astep);
                        const uint64_t bd = bq + (uint64_t)(ks * bkstep);
                        const uint32_t acc = (ks > 0 || i > 0) ? 1u : 0u;
                        umma::mma_s8_warp(tmem + tb * C::BUFC + i * C::NB, ad, bd, idesc[i], acc);
                    }
                }
                umma::commit_warp(&accfull[tb]);
                umma::commit_warp(&bempty[bs]);
            }
            umma::commit_warp(&fin);
        }
    } else {
        // ---- epilogue: atom row = 32 (warp % 4) + lane, column quarter = warp / 4
        const int qd = warp & 3, part = warp >> 2;
        const int r = 32 * qd + lane;
        const int i = tile * 128 + r;
        const double2* sxy = reinterpret_cast<const double2*>(smem + L.xy_off);
        double E[3] = {0, 0, 0}, G[6] = {0, 0, 0, 0, 0, 0}, H[3] = {0, 0, 0}, SI1 = 0, SR2 = 0;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * qd) << 16);
        constexpr int WN = C::WN;
        static_assert(WN == 16 || WN == 12, "a 16-column, or an 8- and a 4-column, load per digit level");
        bool ok = tc_wait(&ares, 0, err, 16, &abort_);
        for (int q = 0; q < ncb && ok; ++q) {
            const int bs = q % NBS, tb = q & 1;
            if (!tc_wait(&accfull[tb], (q >> 1) & 1, err, 32, &abort_)) break;
            umma::fence_after_sync();
            float d[ND][WN];
#pragma unroll
            for (int lv = 0; lv < ND; ++lv) {
                const uint32_t ta = lane_base + tb * C::BUFC + lv * C::NB + part * WN;
                if (WN == 16) {
                    umma::tmem_ld16(ta, d[lv]);
                } else {
                    umma::tmem_ld8(ta, d[lv]);
                    umma::tmem_ld4(ta + 8, d[lv] + 8);
                }
            }
            umma::tmem_wait_ld();
            umma::fence_before_sync();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&accfree[tb]);
            const double* kcst =
                reinterpret_cast<const double*>(smem + L.b_off + bs * L.stage_bytes + (size_t)ND * C::NB * KZ);
#pragma unroll
            for (int cc = 0; cc < C::HC; ++cc) {
                const double* k = kcst + (part * C::HC + cc) * NCONST;
                const int ex = (int)k[14], ey = (int)k[15];
                const double2 X = sxy[ex * 128 + r], Y = sxy[ey * 128 + r];
                const double wr = fma(X.x, Y.x, -X.y * Y.y), wi = fma(X.x, Y.y, X.y * Y.x);
                const int o = cc * NMOM * 2;
                // F_j in true units; the nz = 0 row adds conj(a[c, 0]) to F_0
                const double f0r = fma(k[0], comb4(d[0][o], d[1][o], d[2][o], d[3][o]), k[12]);
                const double f0i = fma(k[0], comb4(d[0][o + 1], d[1][o + 1], d[2][o + 1], d[3][o + 1]), k[13]);
                const double f1r = k[1] * comb4(d[0][o + 2], d[1][o + 2], d[2][o + 2], d[3][o + 2]);
                const double f1i = k[1] * comb4(d[0][o + 3], d[1][o + 3], d[2][o + 3], d[3][o + 3]);
                const double i0 = fma(wr, f0i, wi * f0r), i1 = fma(wr, f1i, wi * f1r);
                E[0] = fma(k[3], i0, E[0]);
                E[1] = fma(k[4], i0, E[1]);
                E[2] = fma(k[5], i0, E[2]);
                SI1 += i1;
                if (NMOM == 3) {
                    const double f2r = k[2] * comb4(d[0][o + 4], d[1][o + 4], d[2][o + 4], d[3][o + 4]);
                    const double f2i = k[2] * comb4(d[0][o + 5], d[1][o + 5], d[2][o + 5], d[3][o + 5]);
                    const double r0 = fma(wr, f0r, -wi * f0i), r1 = fma(wr, f1r, -wi * f1i);
                    const double r2 = fma(wr, f2r, -wi * f2i);
#pragma unroll
                    for (int e = 0; e < 6; ++e) G[e] = fma(k[6 + e], r0, G[e]);
#pragma unroll
                    for (int e = 0; e < 3; ++e) H[e] = fma(k[3 + e], r1, H[e]);
                    SR2 += r2;
                }
            }
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&bempty[bs]);
        }
        if (i < n && !abort_) {
            const double b3[3] = {2.0 * PI * c.B[2], 2.0 * PI * c.B[5], 2.0 * PI * c.B[8]};
            double* o = fpart + (size_t)part * 9 * n;
            for (int dd = 0; dd < 3; ++dd) o[(size_t)dd * n + i] = E[dd] + b3[dd] * SI1;
            if (NMOM == 3) {
                const int pd[6] = {0, 1, 2, 0, 0, 1}, pe[6] = {0, 1, 2, 1, 2, 2};
                for (int e = 0; e < 6; ++e)
                    o[(size_t)(3 + e) * n + i] =
                        G[e] + b3[pe[e]] * H[pd[e]] + b3[pd[e]] * H[pe[e]] + b3[pd[e]] * b3[pe[e]] * SR2;
            }
        }
    }
    // every MMA has completed before the tensor memory is released
    if (warp == 0) tc_wait(&fin, 0, err, 64, &abort_);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace tc4
}  // namespace mdff
