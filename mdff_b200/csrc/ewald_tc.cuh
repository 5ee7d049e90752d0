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
// evaluation by sixteen producer warps from per-atom tables X, Y (FP32, built
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
constexpr int NBUF = 4;                // pipeline depth
constexpr int NPW = 16;                // producer warps (row x 4-atom chunk per thread)
constexpr int THREADS = 32 * (NPW + 2);   // + MMA warp + copy warp
constexpr int LSTRIDE = 160;           // tensor-memory columns per digit level when N > 128 (N <= 160)
constexpr int A_SLICE = 128 * KB;      // bytes of one A digit slice per stage
constexpr uint64_t WAIT_NS = 200000000ull;   // 0.2 s: a pipeline wait longer than this is an error

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
    // the three digit slices side by side along N (rows s N + r), so that
    // one MMA multiplies an A slice by two B slices at once
    const int blk = a / SA, al = a % SA;
    uint8_t* base = img + (size_t)blk * 3 * N * KB;
    const uint32_t lbo = (uint32_t)(3 * N / 8) * 128, sstep = (uint32_t)(N / 8) * 128;
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
        *reinterpret_cast<uint32_t*>(base + sstep + off) = s2;
        *reinterpret_cast<uint32_t*>(base + 2u * sstep + off) = s3;
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

__device__ __forceinline__ bool tc_wait(uint64_t* b, uint32_t parity, int* err, int code, volatile int* stop) {
    if (umma::mbar_wait_ns(b, parity, WAIT_NS, stop)) return true;
    if (!*stop) atomicOr(err, code);
    *stop = 1;
    return false;
}

// grid (tiles, splits); THREADS threads; dynamic shared memory Layout::smem_bytes().
// Q = false when the sources carry no charges (the solver's operator
// applications): the amplitude's real part is zero and its products drop out,
// with the same digits (an FMA with a zero product returns its addend).
template <bool Q>
__global__ void __launch_bounds__(THREADS, 1)
    k_sfac_tc(int nblk, int bps, const uint8_t* __restrict__ bimg, const float2* __restrict__ xy,
              const float4* __restrict__ prm, const float* __restrict__ amax, const int* __restrict__ cols, int nsph,
              int kx, int ky, int kz, int nzl, int N, int XYW, int ncol, size_t plane, double* __restrict__ part_re,
              double* __restrict__ part_im, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[NBUF], aready[NBUF], empty[NBUF], done;
    __shared__ uint32_t tslot;
    __shared__ float red[THREADS / 32];
    __shared__ volatile int stop;
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
        stop = 0;
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
        // ---- producers: row r of the A tile, atoms [4h, 4h + 4) of each stage
        const int r = tid & 127, h = tid >> 7;
        const int li = tile * 128 + r;
        const int col = li < nsph ? cols[li] : -1;
        const int ny_n = 2 * ky + 1;
        const int nx = col >= 0 ? col / ny_n : 0, ny = col >= 0 ? col % ny_n - ky : 0;
        const float rinv = col >= 0 ? inv : 0.f;
        const float fnx = (float)nx * rinv, fny = (float)ny * rinv, gk = (float)kz * rinv;
        const int ex = nx, ey = kx + 1 + ny + ky;
        for (int s = 0; s < nst; ++s) {
            const int b = s % NBUF;
            if (!tc_wait(&full[b], (s / NBUF) & 1, err, 2, &stop)) break;
            uint8_t* bb = smem + b * L.buf_bytes;
            const float2* sxy = reinterpret_cast<const float2*>(bb + L.xy_off);
            const float4* sp = reinterpret_cast<const float4*>(bb + L.p_off);
            {                                      // 4 atoms = one 16-byte chunk per slice
                uint32_t w1[4], w2[4], w3[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int al = 4 * h + u;
                    const float2 X = sxy[al * XYW + ex], Y = sxy[al * XYW + ey];
                    const float4 P = sp[al];
                    const float xr = fmaf(X.x, Y.x, -X.y * Y.y), xi = fmaf(X.x, Y.y, X.y * Y.x);
                    const float ai = fmaf(fnx, P.y, fny * P.z), gg = P.w * gk;
                    float a0r, a0i;
                    if (Q) {
                        const float ar = P.x * rinv;
                        a0r = fmaf(xr, ar, -xi * ai);
                        a0i = fmaf(xr, ai, xi * ar);
                    } else {
                        a0r = -xi * ai;
                        a0i = xr * ai;
                    }
                    const float a1r = xr * gg, a1i = xi * gg;
                    umma::slices4(umma::digits24(__float2int_rn(a0r)), umma::digits24(__float2int_rn(a0i)),
                                  umma::digits24(__float2int_rn(a1r)), umma::digits24(__float2int_rn(a1i)), w1[u],
                                  w2[u], w3[u]);
                }
                const int kc = h;                  // core-matrix column (16 K bytes)
                const uint32_t off = (uint32_t)kc * (16 * 128) + (uint32_t)(r >> 3) * 128 + (r & 7) * 16;
                *reinterpret_cast<uint4*>(bb + L.a_off + off) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
                *reinterpret_cast<uint4*>(bb + L.a_off + A_SLICE + off) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
                *reinterpret_cast<uint4*>(bb + L.a_off + 2 * A_SLICE + off) = make_uint4(w3[0], w3[1], w3[2], w3[3]);
            }
            umma::fence_smem_to_async();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&aready[b]);
        }
    } else if (warp == NPW + 1) {
        // ---- copies: B digit image, X/Y tables and parameters of each stage,
        // as far ahead as the buffers allow
        if (lane == 0) {
            const uint32_t bytes = L.b_bytes() + SA * XYW * 8u + SA * 16u;
            int last = -1;
            for (int s = 0; s < nst; ++s) {
                const int b = s % NBUF, blk = blk0 + s;
                if (s >= NBUF && !tc_wait(&empty[b], ((s / NBUF) - 1) & 1, err, 1, &stop)) break;
                uint8_t* bb = smem + b * L.buf_bytes;
                umma::mbar_arrive_expect_tx(&full[b], bytes);
                umma::bulk_g2s(bb + L.b_off, bimg + (size_t)blk * L.b_bytes(), L.b_bytes(), &full[b]);
                umma::bulk_g2s(bb + L.xy_off, xy + (size_t)blk * SA * XYW, SA * XYW * 8u, &full[b]);
                umma::bulk_g2s(bb + L.p_off, prm + (size_t)blk * SA, SA * 16u, &full[b]);
                last = s;
            }
            // every copy issued has landed before the CTA can exit, also when the
            // pipeline was abandoned on an error (bounded, whatever the stop flag)
            for (int k = max(0, last - NBUF + 1); k <= last; ++k) umma::mbar_wait_ns(&full[k % NBUF], (k / NBUF) & 1, WAIT_NS);
        }
    } else if (lane == 0) {
        // ---- MMA issue: per stage 2 K-steps of 32 x the six digit products.
        // With N <= 128 the levels sit N columns apart and the B slices side
        // by side, so (A0; B0 B1) -> levels 0-1 and (A1; B0 B1) -> levels 1-2
        // are single MMAs of width 2N: four MMAs per K-step, A0 read twice,
        // A1 and A2 once.  Wider N keeps one MMA per product.
        const bool pair = 2 * N <= 256;
        const uint32_t ls = pair ? (uint32_t)N : (uint32_t)LSTRIDE;
        const uint32_t idesc = umma::idesc_s8(128, N), idesc2 = umma::idesc_s8(128, pair ? 2 * N : N);
        const uint32_t lboA = 16 * 128, lboB = (uint32_t)(3 * N / 8) * 128;
        // a shared-memory descriptor is linear in its address field (address
        // >> 4 in the low 14 bits; every address here is below 256 KB), so
        // each operand's descriptor is one base plus a constant offset
        const uint64_t adesc0 = umma::desc_kmajor(sbase + L.a_off, lboA, 128);
        const uint64_t bdesc0 = umma::desc_kmajor(sbase + L.b_off, lboB, 128);
        const uint32_t bstep = L.buf_bytes >> 4, bslice = ((uint32_t)(N / 8) * 128) >> 4;
        uint32_t started = 0;
        for (int s = 0; s < nst; ++s) {
            const int b = s % NBUF;
            if (!tc_wait(&full[b], (s / NBUF) & 1, err, 4, &stop)) break;
            if (!tc_wait(&aready[b], (s / NBUF) & 1, err, 8, &stop)) break;
            umma::fence_after_sync();
            const uint64_t ab = adesc0 + (uint64_t)(b * bstep), bb = bdesc0 + (uint64_t)(b * bstep);
#pragma unroll
            for (int ks = 0; ks < KB / 32; ++ks) {
                const uint64_t bk = bb + (uint64_t)((2 * ks * lboB) >> 4);
                if (pair) {
                    const uint64_t a0 = ab + (uint64_t)((2 * ks * lboA) >> 4);
                    umma::mma_s8(tmem, a0, bk, idesc2, started);
                    umma::mma_s8(tmem + 2 * ls, a0, bk + 2 * bslice, idesc, started);
                    umma::mma_s8(tmem + ls, a0 + (A_SLICE >> 4), bk, idesc2, 1u);
                    umma::mma_s8(tmem + 2 * ls, a0 + ((2 * A_SLICE) >> 4), bk, idesc, 1u);
                    started = 1u;
                } else {
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3 - i; ++j) {
                            const int lvl = i + j;
                            const uint64_t ad = ab + (uint64_t)((i * A_SLICE + 2 * ks * lboA) >> 4);
                            umma::mma_s8(tmem + lvl * ls, ad, bk + j * bslice, idesc, (started >> lvl) & 1u);
                            started |= 1u << lvl;
                        }
                }
            }
            umma::commit(&empty[b]);
        }
        umma::commit(&done);
    }

    // ---- epilogue: warps 0-3 (tensor-memory lane quarters 0-3), row = lane
    if (warp < 4) {
        const bool ok = nst == 0 || tc_wait(&done, 0, err, 16, &stop);
        umma::fence_after_sync();
        const int r = tid;
        const int li = tile * 128 + r;
        const int col = li < nsph ? cols[li] : -1;
        const double osc = (double)sigma / ((double)umma::QS * (double)umma::QS);
        const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
        const uint32_t ls = 2 * N <= 256 ? (uint32_t)N : (uint32_t)LSTRIDE;
        for (int j = 0; j < N / 16; ++j) {
            float d2[16], d3[16], d4[16];
            if (nst > 0) {
                umma::tmem_ld16(lane_base + 16 * j, d2);
                umma::tmem_ld16(lane_base + ls + 16 * j, d3);
                umma::tmem_ld16(lane_base + 2 * ls + 16 * j, d4);
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

// ===========================================================================
// Field pass on the tensor cores (mixed path).
//
// With a[c, nz] = A_k S(k) on the FP32 set and the same factorisation,
//   sum_k k Im(conj(a_k) e^{i k.r_i}) = sum_c [kc Im(W F0) + b3 Im(W F1)],
//   sum_k k k^T Re(conj(a_k) e^{i k.r_i})
//       = sum_c [kc kc^T Re(W F0) + (kc b3^T + b3 kc^T) Re(W F1) + b3 b3^T Re(W F2)],
// W = X_i[nx] Y_i[ny], kc = nx b1 + ny b2 (b_j = 2 pi (column j of B)),
//   F_j[i, c] = sum_nz Z_i[nz] nz^j conj(a[c, nz])          (j = 0, 1 [, 2]).
// F is a complex GEMM: M = 128 atoms of a tile, K = (nz, re/im), N = (column,
// moment, re/im) in blocks of 16 columns (8 with the field gradient); each CTA
// works through an equal share of the (tile, column block) units (FSeg).  As in
// the structure factor the operands are 24-bit fixed point in three int8
// digits with exact S32 accumulation; A (Z of the tile's atoms) is a digit
// image built per position update, B (nz^j conj(a)) is quantised per
// evaluation with one scale per (column, moment).  The contraction over
// columns runs in the epilogue (8 warps: each atom's row is split over two
// warps by column parts) from the accumulators in tensor memory, double
// buffered so the MMAs of the next column block overlap it; FP32 sums are
// flushed to FP64 after every block.
namespace mdff {
namespace tcf {

constexpr int EPW = 8;                   // epilogue warps: 2 per tensor-memory lane quarter
constexpr int NQ = EPW / 4;              // column parts per block (one per epilogue warp of a quarter)
constexpr int THREADS = 32 * (EPW + 2);  // + MMA warp + copy warp
constexpr int NBS = 6;                   // B stages (the epilogue holds a stage until it has read its constants)

constexpr int NCONST = 16;               // floats of per-column constants
constexpr uint64_t WAIT_NS = 200000000ull;

template <int NMOM>
struct Cfg {
    static constexpr int CB = NMOM == 2 ? 16 : 8;   // columns per block
    static constexpr int NB = CB * NMOM * 2;        // GEMM N per block
    static constexpr int HC = CB / NQ;              // columns per epilogue warp
    static constexpr int LV = NB;                   // tensor-memory columns per digit level
    static constexpr int BUFC = 3 * LV;             // per accumulator buffer (two buffers)
};

struct FLayout {
    int KZ, XYW, NB, CB;
    uint32_t a_off, xy_off, b_off, stage_bytes, img_bytes;
    __host__ __device__ static uint32_t up128(uint32_t x) { return (x + 127u) & ~127u; }
    __host__ __device__ FLayout(int KZ_, int XYW_, int NB_, int CB_) : KZ(KZ_), XYW(XYW_), NB(NB_), CB(CB_) {
        a_off = 0;
        xy_off = up128(3u * 128u * KZ);
        b_off = up128(xy_off + (uint32_t)XYW * 128u * 8u);
        img_bytes = 3u * NB * KZ + (uint32_t)CB * NCONST * 4u;   // B digits + per-column constants
        stage_bytes = up128(img_bytes);
    }
    __host__ __device__ uint32_t a_bytes() const { return 3u * 128u * KZ; }
    __host__ __device__ uint32_t xy_bytes() const { return (uint32_t)XYW * 128u * 8u; }
    __host__ __device__ uint32_t smem_bytes() const { return b_off + NBS * stage_bytes + 128u; }
};

// Per position update: the A digit image of each 128-atom tile, rows = atoms,
// K = (nz row m, re/im) of Z_i[nz]; KZ bytes per row (zero past 2 nzl).
__global__ void k_tcf_aimage(int n, int ntile, const uint32_t* __restrict__ fx, int kz, int nzl, int KZ,
                             uint8_t* __restrict__ img) {
    const int nch = KZ / 16;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ntile * 128 * nch) return;
    const int kc = (int)(t % nch);
    const int a = (int)(t / nch);
    const int tile = a / 128, r = a % 128;
    float v[16];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int m = 8 * kc + u;
        double zs = 0.0, zc = 0.0;
        if (a < n && m < nzl) {
            const uint32_t ph = (uint32_t)(m - kz) * fx[2 * n + a];
            sincospi((double)(int)ph * 4.656612873077393e-10, &zs, &zc);
        }
        v[2 * u] = (float)(zc * (double)umma::QS);
        v[2 * u + 1] = (float)(zs * (double)umma::QS);
    }
    uint32_t s1[4], s2[4], s3[4];
#pragma unroll
    for (int g = 0; g < 4; ++g)
        umma::slices4(umma::digits24(__float2int_rn(v[4 * g])), umma::digits24(__float2int_rn(v[4 * g + 1])),
                      umma::digits24(__float2int_rn(v[4 * g + 2])), umma::digits24(__float2int_rn(v[4 * g + 3])),
                      s1[g], s2[g], s3[g]);
    uint8_t* base = img + (size_t)tile * 3 * 128 * KZ;
    const uint32_t off = (uint32_t)kc * (16 * 128) + (uint32_t)(r >> 3) * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(base + off) = make_uint4(s1[0], s1[1], s1[2], s1[3]);
    *reinterpret_cast<uint4*>(base + 128 * KZ + off) = make_uint4(s2[0], s2[1], s2[2], s2[3]);
    *reinterpret_cast<uint4*>(base + 2 * 128 * KZ + off) = make_uint4(s3[0], s3[1], s3[2], s3[3]);
}

// Per position update: X/Y tables of each tile transposed to [tile][entry][128].
__global__ void k_tcf_xyt(int npad, int ntile, const float2* __restrict__ xy, int XYW, float2* __restrict__ xyt) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ntile * 128 * XYW) return;
    const int r = (int)(t % 128);
    const long te = t / 128;
    const int e = (int)(te % XYW), tile = (int)(te / XYW);
    const int a = tile * 128 + r;
    xyt[t] = a < npad ? xy[(size_t)a * XYW + e] : make_float2(0.f, 0.f);
}

// Per evaluation: the B digit image and per-column constants of each column
// block.  Block = one column block, thread = (GEMM row n, 16-byte K chunk).
// Constants per column: kc s0 (3), s1, kc_d kc_e s0 (00 11 22 01 02 12),
// kc s1 (3), s2, X entry, Y entry; s_j = (scale of moment j) 2^16 / QS^2.
template <int NMOM>
__global__ void k_tcf_bimage(int nsph, const int* __restrict__ cols, int kx, int ky, int kz, int nzl, int KZ,
                             const double* __restrict__ aks, int nrect, CellP c, uint8_t* __restrict__ img) {
    using C = Cfg<NMOM>;
    const int nch = KZ / 16;
    const FLayout L(KZ, 0, C::NB, C::CB);
    __shared__ unsigned smax[C::CB * NMOM];
    const int q = blockIdx.x, t = threadIdx.x;
    if (t < C::CB * NMOM) smax[t] = 0u;
    __syncthreads();
    const int n = t / nch, kc = t % nch;
    const int cl = n / (2 * NMOM), j = (n >> 1) % NMOM, part = n & 1;
    const int li = q * C::CB + cl;
    const int col = li < nsph ? cols[li] : -1;
    double br[8], bi[8];   // nz^j conj(a) over the chunk's 8 rows
    float mx = 0.f;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int m = 8 * kc + u;
        br[u] = 0.0; bi[u] = 0.0;
        if (col >= 0 && m < nzl) {
            const double w = j == 0 ? 1.0 : (j == 1 ? (double)(m - kz) : (double)(m - kz) * (double)(m - kz));
            const size_t r = (size_t)col * nzl + m;
            br[u] = w * aks[r];
            bi[u] = -w * aks[nrect + r];
        }
        mx = fmaxf(mx, (float)fmax(fabs(br[u]), fabs(bi[u])));
    }
    if (t < nch * C::NB) atomicMax(&smax[cl * NMOM + j], __float_as_uint(mx * 1.0000002f));
    __syncthreads();
    uint8_t* base = img + (size_t)q * L.stage_bytes;
    if (t < nch * C::NB) {
        const float sg = __uint_as_float(smax[cl * NMOM + j]);
        const double qsc = sg > 0.f ? (double)umma::QS / (double)sg : 0.0;
        float v[16];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            // part re: (Re B, -Im B); part im: (Im B, Re B)
            v[2 * u] = (float)((part ? bi[u] : br[u]) * qsc);
            v[2 * u + 1] = (float)((part ? br[u] : -bi[u]) * qsc);
        }
        uint32_t s1[4], s2[4], s3[4];
#pragma unroll
        for (int g = 0; g < 4; ++g)
            umma::slices4(umma::digits24(__float2int_rn(v[4 * g])), umma::digits24(__float2int_rn(v[4 * g + 1])),
                          umma::digits24(__float2int_rn(v[4 * g + 2])), umma::digits24(__float2int_rn(v[4 * g + 3])),
                          s1[g], s2[g], s3[g]);
        // the three digit slices side by side along N (rows s NB + n), so
        // that one MMA multiplies an A slice by several B slices at once
        const uint32_t lbo = (uint32_t)(3 * C::NB / 8) * 128;
        const uint32_t off = (uint32_t)kc * lbo + (uint32_t)(n >> 3) * 128 + (n & 7) * 16;
        const uint32_t sstep = (uint32_t)(C::NB / 8) * 128;
        *reinterpret_cast<uint4*>(base + off) = make_uint4(s1[0], s1[1], s1[2], s1[3]);
        *reinterpret_cast<uint4*>(base + sstep + off) = make_uint4(s2[0], s2[1], s2[2], s2[3]);
        *reinterpret_cast<uint4*>(base + 2 * sstep + off) = make_uint4(s3[0], s3[1], s3[2], s3[3]);
    }
    if (t < C::CB) {
        float* k = reinterpret_cast<float*>(base + 3 * C::NB * KZ) + t * NCONST;
        const int li2 = q * C::CB + t;
        const int col2 = li2 < nsph ? cols[li2] : -1;
        float cv[NCONST];
#pragma unroll
        for (int e = 0; e < NCONST; ++e) cv[e] = 0.f;
        if (col2 >= 0) {
            const int ny_n = 2 * ky + 1;
            const int nx = col2 / ny_n, ny = col2 % ny_n - ky;
            const double w = 65536.0 / ((double)umma::QS * (double)umma::QS);
            double s[3];
            for (int jj = 0; jj < 3; ++jj) s[jj] = jj < NMOM ? (double)__uint_as_float(smax[t * NMOM + jj]) * w : 0.0;
            double kc3[3];
            for (int d = 0; d < 3; ++d) kc3[d] = 2.0 * PI * (nx * c.B[3 * d] + ny * c.B[3 * d + 1]);
            cv[0] = (float)(kc3[0] * s[0]); cv[1] = (float)(kc3[1] * s[0]); cv[2] = (float)(kc3[2] * s[0]);
            cv[3] = (float)s[1];
            cv[4] = (float)(kc3[0] * kc3[0] * s[0]); cv[5] = (float)(kc3[1] * kc3[1] * s[0]);
            cv[6] = (float)(kc3[2] * kc3[2] * s[0]); cv[7] = (float)(kc3[0] * kc3[1] * s[0]);
            cv[8] = (float)(kc3[0] * kc3[2] * s[0]); cv[9] = (float)(kc3[1] * kc3[2] * s[0]);
            cv[10] = (float)(kc3[0] * s[1]); cv[11] = (float)(kc3[1] * s[1]); cv[12] = (float)(kc3[2] * s[1]);
            cv[13] = (float)s[2];
            cv[14] = __int_as_float(nx);
            cv[15] = __int_as_float(kx + 1 + ny + ky);
        }
#pragma unroll
        for (int e = 0; e < NCONST; ++e) k[e] = cv[e];
    }
}

__device__ __forceinline__ bool f_wait(uint64_t* b, uint32_t parity, int* err, int code, volatile int* abort_) {
    if (umma::mbar_wait_ns(b, parity, WAIT_NS, abort_)) return true;
    if (!*abort_) atomicOr(err, code);
    *abort_ = 1;
    return false;
}

// exact digit-level sums -> FP32: (D0 2^8 + D1) 2^8 + D2 (the common 2^16 and
// the column scale live in the per-column constants)
__device__ __forceinline__ float comb3(float d0, float d1, float d2) {
    const int t = __float_as_int(d0) * 256 + __float_as_int(d1);
    return fmaf((float)t, 256.f, (float)__float_as_int(d2));
}

// The work is ntile x ncb units (128-atom tile, column block).  CTA b of a
// grid of G <= ntile takes the contiguous units [b U, b U + U), U = ceil(
// ntile ncb / G), so every SM gets the same share (one tile per CTA would
// leave a partial second wave) and, as U >= ncb, a tile is split between at
// most two CTAs.  Its units form segments, one per tile it touches; for each
// segment the tile's A image and X/Y table are loaded again once the previous
// segment's MMAs and epilogue reads are done.  A segment that starts at a
// tile's first column block writes column slot 0 of the tile (and zeros slot
// 1 when it covers the whole tile), one that starts inside it slot 1.
struct FSeg {
    int t0, t1, u0, u1, ncb;
    __device__ FSeg(int ntile, int ncb_, int G, int b) : ncb(ncb_) {
        const long T = (long)ntile * ncb_, U = (T + G - 1) / G;
        u0 = (int)min(T, (long)b * U);
        u1 = (int)min(T, (long)b * U + U);
        t0 = u0 / ncb;
        t1 = u1 > u0 ? (u1 - 1) / ncb : t0 - 1;   // no segment when the range is empty
    }
    __device__ int b0(int t) const { return max(u0 - t * ncb, 0); }
    __device__ int b1(int t) const { return min(u1 - t * ncb, ncb); }
};

// grid = FSeg's G CTAs (at most one per tile); THREADS threads; dynamic
// shared memory FLayout::smem_bytes().  Writes fpart[((slot NQ + part) nv +
// component) n + i] for the NQ column parts and the 2 column slots (nv = 3,
// or 9 with the field gradient).
template <int NMOM>
__global__ void __launch_bounds__(THREADS, 1)
    k_kfield_tc(int n, int ntile, int ncb, const uint8_t* __restrict__ aimg, const float2* __restrict__ xyt,
                const uint8_t* __restrict__ bimg, int KZ, int XYW, CellP c, double* __restrict__ fpart,
                int* __restrict__ err) {
    using C = Cfg<NMOM>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t ares, aempty, bfull[NBS], bempty[NBS], accfull[2], accfree[2], fin;
    __shared__ uint32_t tslot;
    __shared__ volatile int abort_;
    const FLayout L(KZ, XYW, C::NB, C::CB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const FSeg S(ntile, ncb, gridDim.x, blockIdx.x);
    if (tid == 0) {
        umma::mbar_init(&ares, 1);
        umma::mbar_init(&aempty, 1 + EPW);   // the MMA warp's commit + every epilogue warp
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
    if (warp == 0) umma::tmem_alloc(&tslot, 512);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t sbase = umma::smem_u32(smem);

    if (warp == EPW + 1) {
        // ---- copies: lane 0 streams the B stages of every segment's column
        // blocks (q counts blocks over the whole range); lane 1 loads each
        // segment's A image and X/Y table once the previous segment is done
        // every copy issued has landed before the CTA can exit, also when the
        // pipeline was abandoned on an error (bounded waits, whatever the flag)
        if (lane == 0) {
            int q = 0, last = -1;
            for (int t = S.t0; t <= S.t1 && !abort_; ++t)
                for (int bl = S.b0(t); bl < S.b1(t); ++bl, ++q) {
                    const int bs = q % NBS;
                    if (q >= NBS && !f_wait(&bempty[bs], ((q / NBS) - 1) & 1, err, 1, &abort_)) break;
                    umma::mbar_arrive_expect_tx(&bfull[bs], L.img_bytes);
                    umma::bulk_g2s(smem + L.b_off + bs * L.stage_bytes, bimg + (size_t)bl * L.stage_bytes,
                                   L.img_bytes, &bfull[bs]);
                    last = q;
                }
            for (int k = max(0, last - NBS + 1); k <= last; ++k) umma::mbar_wait_ns(&bfull[k % NBS], (k / NBS) & 1, WAIT_NS);
        } else if (lane == 1) {
            int last = -1;
            for (int t = S.t0, sg = 0; t <= S.t1; ++t, ++sg) {
                if (sg > 0 && !f_wait(&aempty, (sg - 1) & 1, err, 128, &abort_)) break;
                umma::mbar_arrive_expect_tx(&ares, L.a_bytes() + L.xy_bytes());
                umma::bulk_g2s(smem + L.a_off, aimg + (size_t)t * L.a_bytes(), L.a_bytes(), &ares);
                umma::bulk_g2s(smem + L.xy_off, xyt + (size_t)t * XYW * 128, L.xy_bytes(), &ares);
                last = sg;
            }
            if (last >= 0) umma::mbar_wait_ns(&ares, last & 1, WAIT_NS);
        }
    } else if (warp == EPW) {
        // ---- MMA issue (the whole warp, one elected lane issues): per column
        // block KZ/32 K-steps x 3 MMAs, A digit i times B digits 0..2-i (side
        // by side along N) into levels i..2: the six digit products, each A
        // slice read once per K-step
        {
            const uint32_t idesc[3] = {umma::idesc_s8(128, 3 * C::NB), umma::idesc_s8(128, 2 * C::NB),
                                       umma::idesc_s8(128, C::NB)};
            const uint32_t lboA = 16 * 128, lboB = (uint32_t)(3 * C::NB / 8) * 128;
            // descriptors as one base per operand plus constant offsets (the
            // address field is linear; every address here is below 256 KB)
            const uint64_t adesc0 = umma::desc_kmajor(sbase + L.a_off, lboA, 128);
            const uint64_t bdesc0 = umma::desc_kmajor(sbase + L.b_off, lboB, 128);
            const uint32_t aslice = (128u * KZ) >> 4;
            const uint32_t astep = (2 * lboA) >> 4, bkstep = (2 * lboB) >> 4, bstage = L.stage_bytes >> 4;
            bool ok = true;
            int q = 0;
            for (int t = S.t0, sg = 0; t <= S.t1 && ok; ++t, ++sg) {
                ok = __all_sync(0xffffffffu, f_wait(&ares, sg & 1, err, 2, &abort_));
                umma::fence_after_sync();
                for (int bl = S.b0(t); bl < S.b1(t) && ok; ++bl, ++q) {
                    const int bs = q % NBS, tb = q & 1;
                    ok = __all_sync(0xffffffffu, f_wait(&bfull[bs], (q / NBS) & 1, err, 4, &abort_));
                    if (ok && q >= 2)
                        ok = __all_sync(0xffffffffu, f_wait(&accfree[tb], ((q >> 1) - 1) & 1, err, 8, &abort_));
                    if (!ok) break;
                    umma::fence_after_sync();
                    const uint64_t bq = bdesc0 + (uint64_t)(bs * bstage);
                    for (int ks = 0; ks < KZ / 32; ++ks) {
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const uint64_t ad = adesc0 + (uint64_t)(i * aslice + ks * astep);
                            const uint64_t bd = bq + (uint64_t)(ks * bkstep);
                            const uint32_t acc = (ks > 0 || i > 0) ? 1u : 0u;
                            umma::mma_s8_warp(tmem + tb * C::BUFC + i * C::LV, ad, bd, idesc[i], acc);
                        }
                    }
                    umma::commit_warp(&accfull[tb]);
                    umma::commit_warp(&bempty[bs]);
                }
                // the segment's A image is free once these MMAs are done
                umma::commit_warp(&aempty);
            }
            umma::commit_warp(&fin);
        }
    } else {
        // ---- epilogue: atom row = 32 (warp % 4) + lane, column part = warp / 4
        const int qd = warp & 3, part = warp >> 2;
        const int r = 32 * qd + lane;
        const float2* sxy = reinterpret_cast<const float2*>(smem + L.xy_off);
        const uint32_t lane_base = tmem + ((uint32_t)(32 * qd) << 16);
        constexpr int WN = C::HC * NMOM * 2;   // accumulator columns per warp per level (32 or 24)
        static_assert(WN <= 32 && C::HC * NQ == C::CB, "two 16-column loads per digit level at most");
        bool ok = true;
        int q = 0;
        for (int t = S.t0, sg = 0; t <= S.t1 && ok; ++t, ++sg) {
            const int i = t * 128 + r;
            double E[3] = {0, 0, 0}, G[6] = {0, 0, 0, 0, 0, 0}, H[3] = {0, 0, 0}, SI1 = 0, SR2 = 0;
            ok = __all_sync(0xffffffffu, f_wait(&ares, sg & 1, err, 16, &abort_));
            for (int bl = S.b0(t); bl < S.b1(t) && ok; ++bl, ++q) {
                const int bs = q % NBS, tb = q & 1;
                ok = __all_sync(0xffffffffu, f_wait(&accfull[tb], (q >> 1) & 1, err, 32, &abort_));
                if (!ok) break;
                umma::fence_after_sync();
                float d[3][32];
#pragma unroll
                for (int lv = 0; lv < 3; ++lv)
#pragma unroll
                    for (int h = 0; h < (WN + 15) / 16; ++h)
                        umma::tmem_ld16(lane_base + tb * C::BUFC + lv * C::LV + part * WN + 16 * h, d[lv] + 16 * h);
                umma::tmem_wait_ld();
                umma::fence_before_sync();
                __syncwarp();
                if (lane == 0) umma::mbar_arrive(&accfree[tb]);
                const float* kcst = reinterpret_cast<const float*>(smem + L.b_off + bs * L.stage_bytes + 3 * C::NB * KZ);
                float e0 = 0.f, e1 = 0.f, e2 = 0.f, si1 = 0.f;
                float g[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, h[3] = {0.f, 0.f, 0.f}, sr2 = 0.f;
#pragma unroll
                for (int cc = 0; cc < C::HC; ++cc) {
                    const float* k = kcst + (part * C::HC + cc) * NCONST;
                    const float4 k0 = *reinterpret_cast<const float4*>(k);
                    const int ex = __float_as_int(k[14]), ey = __float_as_int(k[15]);
                    const float2 X = sxy[ex * 128 + r], Y = sxy[ey * 128 + r];
                    const float wr = fmaf(X.x, Y.x, -X.y * Y.y), wi = fmaf(X.x, Y.y, X.y * Y.x);
                    const int o = cc * NMOM * 2;
                    const float f0r = comb3(d[0][o], d[1][o], d[2][o]), f0i = comb3(d[0][o + 1], d[1][o + 1], d[2][o + 1]);
                    const float f1r = comb3(d[0][o + 2], d[1][o + 2], d[2][o + 2]);
                    const float f1i = comb3(d[0][o + 3], d[1][o + 3], d[2][o + 3]);
                    const float i0 = fmaf(wr, f0i, wi * f0r), i1 = fmaf(wr, f1i, wi * f1r);
                    e0 = fmaf(k0.x, i0, e0);
                    e1 = fmaf(k0.y, i0, e1);
                    e2 = fmaf(k0.z, i0, e2);
                    si1 = fmaf(k0.w, i1, si1);
                    if (NMOM == 3) {
                        const float f2r = comb3(d[0][o + 4], d[1][o + 4], d[2][o + 4]);
                        const float f2i = comb3(d[0][o + 5], d[1][o + 5], d[2][o + 5]);
                        const float r0 = fmaf(wr, f0r, -wi * f0i), r1 = fmaf(wr, f1r, -wi * f1i);
                        const float r2 = fmaf(wr, f2r, -wi * f2i);
                        const float4 k1 = *reinterpret_cast<const float4*>(k + 4);
                        const float4 k2 = *reinterpret_cast<const float4*>(k + 8);
                        const float4 k3 = *reinterpret_cast<const float4*>(k + 12);
                        g[0] = fmaf(k1.x, r0, g[0]); g[1] = fmaf(k1.y, r0, g[1]); g[2] = fmaf(k1.z, r0, g[2]);
                        g[3] = fmaf(k1.w, r0, g[3]); g[4] = fmaf(k2.x, r0, g[4]); g[5] = fmaf(k2.y, r0, g[5]);
                        h[0] = fmaf(k2.z, r1, h[0]); h[1] = fmaf(k2.w, r1, h[1]); h[2] = fmaf(k3.x, r1, h[2]);
                        sr2 = fmaf(k3.y, r2, sr2);
                    }
                }
                __syncwarp();
                if (lane == 0) umma::mbar_arrive(&bempty[bs]);
                E[0] += e0; E[1] += e1; E[2] += e2; SI1 += si1;
                if (NMOM == 3) {
                    for (int e = 0; e < 6; ++e) G[e] += g[e];
                    for (int e = 0; e < 3; ++e) H[e] += h[e];
                    SR2 += sr2;
                }
            }
            // the segment's X/Y table is no longer read
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&aempty);
            if (ok && i < n && !abort_) {
                const double b3[3] = {2.0 * PI * c.B[2], 2.0 * PI * c.B[5], 2.0 * PI * c.B[8]};
                const int nv = NMOM == 3 ? 9 : 3;
                const int slot = S.b0(t) > 0 ? 1 : 0;
                double* o = fpart + (size_t)(slot * NQ + part) * nv * n;
                for (int dd = 0; dd < 3; ++dd) o[(size_t)dd * n + i] = E[dd] + b3[dd] * SI1;
                if (NMOM == 3) {
                    const int pd[6] = {0, 1, 2, 0, 0, 1}, pe[6] = {0, 1, 2, 1, 2, 2};
                    for (int e = 0; e < 6; ++e)
                        o[(size_t)(3 + e) * n + i] =
                            G[e] + b3[pe[e]] * H[pd[e]] + b3[pd[e]] * H[pe[e]] + b3[pd[e]] * b3[pe[e]] * SR2;
                }
                if (slot == 0 && S.b1(t) == ncb) {   // the whole tile here: its slot 1 is empty
                    double* z = fpart + (size_t)(NQ + part) * nv * n;
                    for (int k = 0; k < nv; ++k) z[(size_t)k * n + i] = 0.0;
                }
            }
        }
    }
    // every MMA has completed before the tensor memory is released
    if (warp == 0) f_wait(&fin, 0, err, 64, &abort_);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 512);
    }
}

}  // namespace tcf
}  // namespace mdff
