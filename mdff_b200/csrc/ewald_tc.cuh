// Reciprocal-space structure factor on the tensor cores (mixed path).
//
// The phase factorises exactly over the reciprocal-lattice indices,
//   e^{i k.r_a} = X_a[nx] Y_a[ny] Z_a[nz],  X_a[n] = e^{2 pi i n s1_a} (and
// s2, s3 for Y, Z), and the source amplitude is linear in k:
//   q_a + i k.mu_a = q_a + i (nx m1_a + ny m2_a + nz m3_a),  m_j = 2 pi b_j.mu.
// So for a column c = (nx, ny) and row nz,
//   S[c, nz] = sum_a A0[c,a] Z_a[nz] + sum_a A1[c,a] (i nz/kz) Z_a[nz],
//   A0 = X Y (q + i (nx m1 + ny m2)),  A1 = X Y m3 kz,
// a complex GEMM over the atoms: rows = sphere columns (128 per CTA tile),
// N = (nz, re/im), K = (atom, A0 re, A0 im, A1 re, A1 im) in the real
// embedding  Re D = Re A Re B - Im A Im B,  Im D = Re A Im B + Im A Re B.
//
// Precision: every operand value (scaled to |v| <= 1) is a 24-bit fixed-point
// integer split into three signed 8-bit digits, and the six digit products
// with weight >= 2^16 (of 2^32 for the leading pair) run as tcgen05
// kind::i8 MMAs into three S32 accumulators in tensor memory, one per digit
// weight.  Integer accumulation is exact (no rounding at all along K); the
// error is the 24-bit quantisation of the inputs (6e-8 of the scale) and the
// dropped low digit products (below 2^-23 of the scale per term, unbiased) --
// FP32-grade, and independent of the number of atoms summed.
//
// Operands.  B (Z and i (nz/kz) Z) depends on the positions only: its digit
// image is built once per position update in exactly the shared-memory
// layout of a stage and streamed in by plain bulk copies.  A is generated per
// evaluation by eight producer warps from per-atom tables X, Y (FP32, built
// per position update from the exact fixed-point phase in FP64) and the
// per-atom source parameters.  One thread issues the MMAs.  Each CTA covers
// one 128-column tile and one contiguous range of atoms; its accumulators are
// converted to FP64 and written as the same per-split partials the FP32 path
// writes, so k_sfac_reduce forms A_k S(k), energy and stress unchanged.
#include "umma.cuh"

namespace mdff {
namespace tcs {

constexpr int SA = 16;                 // atoms per pipeline stage
constexpr int KB = 4 * SA;             // K bytes per operand row per stage
constexpr int NBUF = 3;                // pipeline depth
constexpr int NPW = 8;                 // producer warps
constexpr int THREADS = 32 * (NPW + 1);
constexpr int LSTRIDE = 160;           // tensor-memory columns per digit level (N <= 160)
constexpr int A_SLICE = 128 * KB;      // bytes of one A digit slice per stage
constexpr uint32_t WAIT_LIMIT = 1u << 22;

struct Layout {
    int N, XYW;
    uint32_t a_off, b_off, xy_off, p_off, buf_bytes;
    __host__ __device__ static uint32_t up128(uint32_t x) { return (x + 127u) & ~127u; }
    __host__ __device__ Layout(int N_, int XYW_) : N(N_), XYW(XYW_) {
        a_off = 0;
        b_off = up128(a_off + 3u * A_SLICE);
        xy_off = up128(b_off + 3u * (uint32_t)N * KB);
        p_off = up128(xy_off + (uint32_t)SA * XYW * 8u);
        buf_bytes = up128(p_off + (uint32_t)SA * 16u);
    }
    __host__ __device__ uint32_t b_bytes() const { return 3u * (uint32_t)N * KB; }
    __host__ __device__ uint32_t smem_bytes() const { return NBUF * buf_bytes + 128u; }
};

// Per position update: X_a[nx] (nx = 0..kx) then Y_a[ny] (ny = -ky..ky) per
// atom, padded to XYW entries; atoms past n get (1, 0).
__global__ void k_tc_xy(int n, int npad, const uint32_t* __restrict__ fx, int kx, int ky, int XYW,
                        float2* __restrict__ xy) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)npad * XYW) return;
    const int a = (int)(t / XYW), e = (int)(t % XYW);
    float2 v = make_float2(0.f, 0.f);
    if (a >= n) {
        v = make_float2(1.f, 0.f);
    } else if (e <= kx) {
        const uint32_t ph = (uint32_t)e * fx[a];
        double s, c;
        sincospi((double)(int)ph * 4.656612873077393e-10, &s, &c);
        v = make_float2((float)c, (float)s);
    } else if (e <= kx + 1 + 2 * ky) {
        const int ny = e - (kx + 1) - ky;
        const uint32_t ph = (uint32_t)ny * fx[n + a];
        double s, c;
        sincospi((double)(int)ph * 4.656612873077393e-10, &s, &c);
        v = make_float2((float)c, (float)s);
    }
    xy[t] = v;
}

// Per position update: the B digit image.  One thread per (atom, nz row m):
// rows 2m (re) and 2m+1 (im) of the four K entries of the atom, in the
// K-major core-matrix layout of one stage (block of SA atoms).
__global__ void k_tc_bimage(int n, int npad, const uint32_t* __restrict__ fx, int kz, int nzl, int N,
                            uint8_t* __restrict__ img) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int half = N / 2;
    if (t >= (long)npad * half) return;
    const int a = (int)(t / half), m = (int)(t % half);
    double b[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // re-row K0..3, im-row K0..3
    if (a < n && m < nzl) {
        const int nz = m - kz;
        const uint32_t ph = (uint32_t)nz * fx[2 * n + a];
        double zs, zc;
        sincospi((double)(int)ph * 4.656612873077393e-10, &zs, &zc);
        const double f = kz > 0 ? (double)nz / (double)kz : 0.0;
        const double b1r = -f * zs, b1i = f * zc;     // i (nz/kz) Z
        b[0] = zc;  b[1] = -zs; b[2] = b1r; b[3] = -b1i;
        b[4] = zs;  b[5] = zc;  b[6] = b1i; b[7] = b1r;
    }
    const int blk = a / SA, al = a % SA;
    uint8_t* base = img + (size_t)blk * 3 * N * KB;
    const uint32_t lbo = (uint32_t)(N / 8) * 128;
#pragma unroll
    for (int row = 0; row < 2; ++row) {
        const int r = 2 * m + row;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = umma::digits24(__double2int_rn(b[4 * row + j] * (double)umma::QS));
        uint32_t s1, s2, s3;
        umma::slices4(w[0], w[1], w[2], w[3], s1, s2, s3);
        const uint32_t off = (uint32_t)(al >> 2) * lbo + (uint32_t)(r >> 3) * 128 + (r & 7) * 16 + 4 * (al & 3);
        *reinterpret_cast<uint32_t*>(base + off) = s1;
        *reinterpret_cast<uint32_t*>(base + (uint32_t)N * KB + off) = s2;
        *reinterpret_cast<uint32_t*>(base + 2u * N * KB + off) = s3;
    }
}

// Per evaluation: (q, m1, m2, m3) per atom and the bound
// max(|q| + kx |m1| + ky |m2|, kz |m3|) of the scaled amplitudes.
__global__ void k_tc_params(int n, int npad, const double* __restrict__ q, const double* __restrict__ mu, CellP c,
                            int with_q, int with_mu, int kx, int ky, int kz, float4* __restrict__ prm,
                            float* __restrict__ amax) {
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
    prm[a] = make_float4((float)qa, (float)m1, (float)m2, (float)m3);
    amax[a] = (float)fmax(fabs(qa) + kx * fabs(m1) + ky * fabs(m2), kz * fabs(m3));
}

__device__ __forceinline__ bool tc_wait(uint64_t* b, uint32_t parity, int* err, int code) {
    if (umma::mbar_wait(b, parity, WAIT_LIMIT)) return true;
    atomicOr(err, code);
    return false;
}

// grid (tiles, splits); THREADS threads; dynamic shared memory Layout::smem_bytes().
__global__ void __launch_bounds__(THREADS, 1)
    k_sfac_tc(int nblk, int bps, const uint8_t* __restrict__ bimg, const float2* __restrict__ xy,
              const float4* __restrict__ prm, const float* __restrict__ amax, const int* __restrict__ cols, int nsph,
              int kx, int ky, int kz, int nzl, int N, int XYW, int ncol, size_t plane, double* __restrict__ part_re,
              double* __restrict__ part_im, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[NBUF], aready[NBUF], empty[NBUF], done;
    __shared__ uint32_t tslot;
    __shared__ float red[THREADS / 32];
    const Layout L(N, XYW);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x, split = blockIdx.y;
    const int blk0 = split * bps, blk1 = min(nblk, blk0 + bps);
    const int nst = max(0, blk1 - blk0);

    // the scale of this CTA's atoms
    float mx = 0.f;
    for (int a = blk0 * SA + tid; a < blk1 * SA; a += THREADS) mx = fmaxf(mx, amax[a]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) {
            umma::mbar_init(&full[b], 1);
            umma::mbar_init(&aready[b], NPW);
            umma::mbar_init(&empty[b], 1);
        }
        umma::mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) umma::tmem_alloc(&tslot, 512);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    float sigma = 0.f;
    for (int w = 0; w < THREADS / 32; ++w) sigma = fmaxf(sigma, red[w]);
    sigma = fmaxf(sigma, 1e-30f);
    const float inv = umma::QS / sigma;
    const uint32_t sbase = umma::smem_u32(smem);

    if (warp < NPW) {
        // ---- producers: row r of the A tile, atoms [8h, 8h + 8) of each stage
        const int r = tid & 127, h = tid >> 7;
        const int li = tile * 128 + r;
        const int col = li < nsph ? cols[li] : -1;
        const int ny_n = 2 * ky + 1;
        const int nx = col >= 0 ? col / ny_n : 0, ny = col >= 0 ? col % ny_n - ky : 0;
        const float rinv = col >= 0 ? inv : 0.f;
        const float fnx = (float)nx * rinv, fny = (float)ny * rinv, gk = (float)kz * rinv;
        const int ex = nx, ey = kx + 1 + ny + ky;
        bool ok = true;
        for (int s = 0; s < nst && ok; ++s) {
            const int b = s % NBUF;
            if (tid == 0 && s == 0) {
                const int blk = blk0;
                umma::mbar_arrive_expect_tx(&full[0], L.b_bytes() + SA * XYW * 8u + SA * 16u);
                umma::bulk_g2s(smem + L.b_off, bimg + (size_t)blk * L.b_bytes(), L.b_bytes(), &full[0]);
                umma::bulk_g2s(smem + L.xy_off, xy + (size_t)blk * SA * XYW, SA * XYW * 8u, &full[0]);
                umma::bulk_g2s(smem + L.p_off, prm + (size_t)blk * SA, SA * 16u, &full[0]);
            }
            if (tid == 0 && s + 1 < nst) {
                const int bn = (s + 1) % NBUF, blk = blk0 + s + 1;
                if (s + 1 >= NBUF && !tc_wait(&empty[bn], ((s + 1) / NBUF - 1) & 1, err, 1)) ok = false;
                uint8_t* bb = smem + bn * L.buf_bytes;
                umma::mbar_arrive_expect_tx(&full[bn], L.b_bytes() + SA * XYW * 8u + SA * 16u);
                umma::bulk_g2s(bb + L.b_off, bimg + (size_t)blk * L.b_bytes(), L.b_bytes(), &full[bn]);
                umma::bulk_g2s(bb + L.xy_off, xy + (size_t)blk * SA * XYW, SA * XYW * 8u, &full[bn]);
                umma::bulk_g2s(bb + L.p_off, prm + (size_t)blk * SA, SA * 16u, &full[bn]);
            }
            if (!tc_wait(&full[b], (s / NBUF) & 1, err, 2)) { ok = false; break; }
            uint8_t* bb = smem + b * L.buf_bytes;
            const float2* sxy = reinterpret_cast<const float2*>(bb + L.xy_off);
            const float4* sp = reinterpret_cast<const float4*>(bb + L.p_off);
#pragma unroll
            for (int g = 0; g < 2; ++g) {          // two groups of 4 atoms = one 16-byte chunk each
                uint32_t w1[4], w2[4], w3[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int al = 8 * h + 4 * g + u;
                    const float2 X = sxy[al * XYW + ex], Y = sxy[al * XYW + ey];
                    const float4 P = sp[al];
                    const float xr = fmaf(X.x, Y.x, -X.y * Y.y), xi = fmaf(X.x, Y.y, X.y * Y.x);
                    const float ar = P.x * rinv, ai = fmaf(fnx, P.y, fny * P.z), gg = P.w * gk;
                    const float a0r = fmaf(xr, ar, -xi * ai), a0i = fmaf(xr, ai, xi * ar);
                    const float a1r = xr * gg, a1i = xi * gg;
                    umma::slices4(umma::digits24(__float2int_rn(a0r)), umma::digits24(__float2int_rn(a0i)),
                                  umma::digits24(__float2int_rn(a1r)), umma::digits24(__float2int_rn(a1i)), w1[u],
                                  w2[u], w3[u]);
                }
                const int kc = 2 * h + g;          // core-matrix column (16 K bytes)
                const uint32_t off = (uint32_t)kc * (16 * 128) + (uint32_t)(r >> 3) * 128 + (r & 7) * 16;
                *reinterpret_cast<uint4*>(bb + L.a_off + off) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
                *reinterpret_cast<uint4*>(bb + L.a_off + A_SLICE + off) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
                *reinterpret_cast<uint4*>(bb + L.a_off + 2 * A_SLICE + off) = make_uint4(w3[0], w3[1], w3[2], w3[3]);
            }
            umma::fence_smem_to_async();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&aready[b]);
        }
    } else if (lane == 0) {
        // ---- MMA issue: per stage 2 K-steps of 32 x 6 digit products
        const uint32_t idesc = umma::idesc_s8(128, N);
        const uint32_t lboA = 16 * 128, lboB = (uint32_t)(N / 8) * 128;
        uint32_t started = 0;
        for (int s = 0; s < nst; ++s) {
            const int b = s % NBUF;
            if (!tc_wait(&full[b], (s / NBUF) & 1, err, 4)) break;
            if (!tc_wait(&aready[b], (s / NBUF) & 1, err, 8)) break;
            umma::fence_after_sync();
            const uint32_t a0 = sbase + b * L.buf_bytes + L.a_off, b0 = sbase + b * L.buf_bytes + L.b_off;
#pragma unroll
            for (int ks = 0; ks < KB / 32; ++ks) {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3 - i; ++j) {
                        const int lvl = i + j;
                        const uint64_t ad = umma::desc_kmajor(a0 + i * A_SLICE + 2 * ks * lboA, lboA, 128);
                        const uint64_t bd = umma::desc_kmajor(b0 + j * (uint32_t)N * KB + 2 * ks * lboB, lboB, 128);
                        umma::mma_s8(tmem + lvl * LSTRIDE, ad, bd, idesc, (started >> lvl) & 1u);
                        started |= 1u << lvl;
                    }
            }
            umma::commit(&empty[b]);
        }
        umma::commit(&done);
    }

    // ---- epilogue: warps 0-3 (tensor-memory lane quarters 0-3), row = lane
    if (warp < 4) {
        const bool ok = nst == 0 || tc_wait(&done, 0, err, 16);
        umma::fence_after_sync();
        const int r = tid;
        const int li = tile * 128 + r;
        const int col = li < nsph ? cols[li] : -1;
        const double osc = (double)sigma / ((double)umma::QS * (double)umma::QS);
        const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
        for (int j = 0; j < N / 16; ++j) {
            float d2[16], d3[16], d4[16];
            if (nst > 0) {
                umma::tmem_ld16(lane_base + 16 * j, d2);
                umma::tmem_ld16(lane_base + LSTRIDE + 16 * j, d3);
                umma::tmem_ld16(lane_base + 2 * LSTRIDE + 16 * j, d4);
                umma::tmem_wait_ld();
            }
            if (col < 0 || !ok) continue;
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int nn = 16 * j + e, m = nn >> 1;
                if (m >= nzl) continue;
                double v = 0.0;
                if (nst > 0)
                    v = ((double)__float_as_int(d2[e]) * 4294967296.0 + (double)__float_as_int(d3[e]) * 16777216.0 +
                         (double)__float_as_int(d4[e]) * 65536.0) * osc;
                const size_t idx = (size_t)split * plane + (size_t)m * ncol + col;
                if (nn & 1) part_im[idx] = v;
                else part_re[idx] = v;
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 512);
    }
}

}  // namespace tcs
}  // namespace mdff
