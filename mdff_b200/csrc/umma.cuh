// Fifth-generation tensor core (tcgen05) helpers for sm_100a: shared-memory
// matrix descriptors, the instruction descriptor of kind::f16 (BF16 inputs,
// FP32 accumulator in tensor memory), MMA issue and commit, tensor-memory
// allocation and loads, and bounded mbarrier waits.  Inline PTX only.
//
// Operand layout (both operands K-major, no swizzle): an R x K tile is a grid
// of 8-row x 16-byte "core matrices" (8 rows of 8 BF16 each, 128 contiguous
// bytes).  Element (r, k) sits at
//     (k / 8) * LBO + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// with LBO = (R / 8) * 128 the distance between core matrices adjacent in K
// and SBO = 128 the distance between core matrices adjacent in R.  One MMA
// with K = 16 reads the two K-adjacent core-matrix columns starting at its
// descriptor's address.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace mdff {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of a K-major, no-swizzle tile with R rows
__host__ __device__ __forceinline__ uint32_t kmajor_off(int R, int r, int k) {
    return (uint32_t)((k >> 3) * (R >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading (K) and stride
// (8-row group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 D
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// instruction descriptor of kind::i8: signed 8-bit A and B (both K-major),
// S32 D.  The integer products and sums are exact.
__host__ __device__ constexpr uint32_t idesc_s8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// byte offset of element (r, k) of a K-major, no-swizzle 8-bit tile with R
// rows (core matrices of 8 rows x 16 elements)
__host__ __device__ __forceinline__ uint32_t kmajor_off_i8(int R, int r, int k) {
    return (uint32_t)((k >> 4) * (R >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 15));
}

// D (tensor memory) = A B^T (+ D when acc != 0); issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// D (tensor memory, S32) = A B^T (+ D when acc != 0), signed 8-bit operands
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// arrive on the mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

// The same two, called by a whole converged warp with warp-uniform operands;
// one elected lane issues.  Beside warps doing FP32 work on the same
// scheduler, a single issuing thread in a divergent branch is starved of issue
// slots (every MMA needs its operands moved to uniform registers first) and
// the tensor pipe idles between its MMAs; a warp-uniform loop keeps the
// descriptors in uniform registers and needs a few issue slots per MMA.
__device__ __forceinline__ void mma_s8_warp(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred e, p;\n\telect.sync _|e, 0xffffffff;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void commit_warp(uint64_t* mbar) {
    asm volatile(
        "{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(smem_u32(mbar))
        : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// tensor-memory allocation (one full warp); the address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 columns of 32-bit words: thread t of the warp receives lane
// (lane field of taddr) + t, columns col .. col + 15.  A warp may only touch
// the 32-lane quarter (warp id % 4) of tensor memory.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v) {
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// announce `bytes` of asynchronous copies completing on this phase, and arrive
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// plain (non-multicast) bulk copy global -> this CTA's shared memory; both
// addresses 16-byte aligned, size a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(mbar))
        : "memory");
}

// Wait for phase `parity` of the mbarrier to complete; gives up after
// `limit` polls (about limit * 64 ns) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_test(b, parity)) return true;
        if (it > 32) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// try_wait suspends the warp in hardware until the phase completes or a
// short system-defined limit passes, so waiting costs almost no issue slots
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait by elapsed time: false once `limit_ns` has passed (or *stop
// became nonzero) without the phase completing.
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* b, uint32_t parity, uint64_t limit_ns,
                                             const volatile int* stop = nullptr) {
    if (mbar_try(b, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_try(b, parity)) {
        if (stop && *stop) return false;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
    return true;
}

// Two FP32 values as one BF16 pair (round to nearest): e0 in the low half
// (lower address, even K index), e1 in the high half.
__device__ __forceinline__ uint32_t pack_bf16x2(float e0, float e1) {
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(e1), "f"(e0));
    return d;
}
__device__ __forceinline__ float bf16_lo(uint32_t d) { return __uint_as_float(d << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t d) { return __uint_as_float(d & 0xFFFF0000u); }

// Three round-to-nearest BF16 slices of a pair: e = s0 + s1 + s2 to about
// 2^-24 relative (each residual is exact in FP32).
__device__ __forceinline__ void split3_bf16x2(float e0, float e1, uint32_t& s0, uint32_t& s1, uint32_t& s2) {
    s0 = pack_bf16x2(e0, e1);
    e0 -= bf16_lo(s0);
    e1 -= bf16_hi(s0);
    s1 = pack_bf16x2(e0, e1);
    e0 -= bf16_lo(s1);
    e1 -= bf16_hi(s1);
    s2 = pack_bf16x2(e0, e1);
}

// ---- 24-bit fixed point in three signed 8-bit slices ------------------------
// V = rn(v * QS) with |V| <= 0x7F7F7F; the bytes of (V + 0x808080) ^ 0x808080
// are signed digits d1 (byte 2, most significant), d2, d3 with
// V = d1 2^16 + d2 2^8 + d3, d1 in [-127, 127], d2, d3 in [-128, 127].
constexpr float QS = 8355000.f;
__device__ __forceinline__ uint32_t digits24(int V) { return ((uint32_t)V + 0x808080u) ^ 0x808080u; }
// Four values (consecutive K) -> one 32-bit word per slice: s1 (most
// significant digits) .. s3.
__device__ __forceinline__ void slices4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t& s1, uint32_t& s2,
                                        uint32_t& s3) {
    const uint32_t t01 = __byte_perm(w0, w1, 0x5140), t23 = __byte_perm(w2, w3, 0x5140);
    s3 = __byte_perm(t01, t23, 0x5410);
    s2 = __byte_perm(t01, t23, 0x7632);
    const uint32_t v01 = __byte_perm(w0, w1, 0x0062), v23 = __byte_perm(w2, w3, 0x0062);
    s1 = __byte_perm(v01, v23, 0x5410);
}

// ---- 32-bit fixed point in four signed 8-bit slices --------------------------
// V = rn(v * QS4) with |V| <= 0x7F7F7F7F; the bytes of (V + 0x80808080) ^
// 0x80808080 are signed digits d1 (byte 3, most significant) .. d4 with
// V = d1 2^24 + d2 2^16 + d3 2^8 + d4, d1 in [-127, 127], the others in
// [-128, 127].  QS4 leaves 2.9e-5 of headroom for |v| <= 1 plus rounding.
constexpr double QS4 = 2139000000.0;
__device__ __forceinline__ uint32_t digits32(int V) { return ((uint32_t)V + 0x80808080u) ^ 0x80808080u; }
// Four values (consecutive K) -> one 32-bit word per slice: s1 (most
// significant digits) .. s4.
__device__ __forceinline__ void slices4x4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t& s1,
                                          uint32_t& s2, uint32_t& s3, uint32_t& s4) {
    const uint32_t t01 = __byte_perm(w0, w1, 0x5140), t23 = __byte_perm(w2, w3, 0x5140);   // bytes 0 and 1
    const uint32_t u01 = __byte_perm(w0, w1, 0x7362), u23 = __byte_perm(w2, w3, 0x7362);   // bytes 2 and 3
    s4 = __byte_perm(t01, t23, 0x5410);
    s3 = __byte_perm(t01, t23, 0x7632);
    s2 = __byte_perm(u01, u23, 0x5410);
    s1 = __byte_perm(u01, u23, 0x7632);
}

// Conversions on the FP64 pipe instead of the conversion unit: 1.5 * 2^52
// has a unit in the last place of 1, so v + M rounds v to the nearest
// integer (ties to even, as cvt.rni) and its low word is that integer for
// |v| < 2^31; and the bit pattern of M plus an integer |x| < 2^51 is the
// double M + x, from which M subtracts exactly.
constexpr double MAGIC52 = 6755399441055744.0;
__device__ __forceinline__ int rint_i32(double v) { return __double2loint(v + MAGIC52); }
__device__ __forceinline__ double i64_to_f64(long long x) {
    return __longlong_as_double(0x4338000000000000ll + x) - MAGIC52;
}

}  // namespace umma
}  // namespace mdff
