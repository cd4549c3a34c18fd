// Thin inline-PTX wrappers for the sm_100a pieces the ensemble kernel uses:
// tensor memory (TMEM) allocation, tcgen05.mma kind::tf32 and kind::f16 (BF16 or FP16)
// with shared-memory operands, tcgen05.commit to an mbarrier, tcgen05.ld of the accumulator, and
// bounded mbarrier waits.  Descriptor formats follow the PTX ISA's tcgen05
// "shared memory descriptor" and "instruction descriptor" tables.
#pragma once

#include <cstdint>

namespace swe {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- TMEM -------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- descriptors --------------------------------------------------------------------
// Shared-memory matrix descriptor, no swizzle (canonical K-major "interleave"
// layout: 8-row x 16-byte core matrices; lbo = byte step between core
// matrices along K, sbo = byte step between 8-row groups along M/N).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor for kind::tf32, FP32 accumulator, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4)                 // D format F32
           | (2u << 7)               // A format TF32
           | (2u << 10)              // B format TF32
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Instruction descriptor for kind::f16 with BF16 A and B (the same type, as kind::f16
// requires), FP32 accumulator, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4)                 // D format F32
           | (1u << 7)               // A format BF16
           | (1u << 10)              // B format BF16
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Instruction descriptor for kind::f16 with FP16 A and B, FP32 accumulator, both
// operands K-major (A and B formats 0 = F16).
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
    return (1u << 4)                 // D format F32
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem], BF16 or FP16 operands (one type for both), K = 16
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int t = 0; t < 16; ++t) v[t] = __uint_as_float(r[t]);
}
// 16 lanes x 256 bits, 4 times along the columns (32 columns): thread i gets lanes
// l = i / 4 and l + 8 of the 16 starting at taddr's lane, columns 8 k + 2 (i % 4) + b:
// v[4 k + b] from lane l, v[4 k + 2 + b] from lane l + 8 (k = 0..3, b = 0, 1)
__device__ __forceinline__ void tmem_ld16x256(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int t = 0; t < 16; ++t) v[t] = __uint_as_float(r[t]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- mbarrier -----------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// try_wait with a suspend-time hint: a thread whose phase is not complete sleeps in
// hardware until it completes or about `hint_ns` pass, instead of re-polling.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* b, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Time-bounded wait that sleeps between tries (see mbar_try_wait_hint); false once
// limit_ns of wall time have passed without the phase completing.
__device__ __forceinline__ bool mbar_wait_timed(uint64_t* b, uint32_t parity, uint64_t limit_ns,
                                                uint32_t hint_ns = 20000) {
    if (mbar_try_wait(b, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait_hint(b, parity, hint_ns)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// Bounded wait: gives up after max_tries polls (each try_wait already
// suspends for a hardware-defined interval); returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, uint32_t max_tries) {
    for (uint32_t t = 0; t < max_tries; ++t)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}

// ---- bulk copies (global -> shared, completion counted in bytes on an mbarrier) ------
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(tx) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(mbar))
        : "memory");
}

// Round an FP32 value to the nearest TF32 (10 explicit mantissa bits), ties
// away from zero; the result is exactly representable, so the tensor core's
// own FP32 -> TF32 conversion leaves it unchanged.
// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away from zero,
// for finite x: half a TF32 ulp is added to the magnitude bits and the 13 bits below
// the TF32 mantissa are cleared (a carry out of the mantissa moves the exponent up,
// which is the correctly rounded result).  Two full-rate integer operations, which
// the operand converters issue for every element they split.
__device__ __forceinline__ float tf32_rna(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}
// 3xTF32 split with lo left in FP32: hi = tf32_rna(x) and lo = x - hi exactly (hi has
// 11 significant bits, so x - hi is representable).  The tensor core reads lo at TF32
// precision (its low 13 bits dropped): |x - hi - lo_used| <= 2^-10 |lo| <= 2^-21 |x|.
__device__ __forceinline__ void tf32_split_lo_fp32(float x, float& hi, float& lo) {
    hi = tf32_rna(x);
    lo = x - hi;
}
// 3xTF32 split x ~ hi + lo with both parts exact TF32: |x - hi - lo| <= 2^-22 |x|.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - hi);
}

}  // namespace tc
}  // namespace swe
