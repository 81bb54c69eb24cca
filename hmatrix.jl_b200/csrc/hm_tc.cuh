// Blackwell (sm_100a) primitives for the tensor-core kernels: shared-memory
// descriptors and the 5th-generation MMA (tcgen05) with its tensor memory
// (TMEM) accumulators, mbarriers, cp.async gathers and 1-D bulk (TMA engine)
// copies.  Inline PTX only; every wait is bounded and reports a timeout
// instead of spinning forever.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hm {
namespace tc {

// ---------------------------------------------------------------------------
// addresses, fences, mbarriers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}

// one arrival that also announces `bytes` of asynchronous copies
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of `parity` to complete; gives up after `limit` polls
// (each try_wait itself suspends for a while) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = (1u << 22)) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---------------------------------------------------------------------------
// cp.async (Ampere-style gathers, 16 or 4 bytes, zero-filled beyond src_bytes)
// and the 1-D bulk copy of the TMA engine
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// one arrival on `bar` once every cp.async issued so far by this thread has
// landed (the barrier's expected count includes it: .noinc)
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned;
// completion is counted on `bar` (complete_tx)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// ---------------------------------------------------------------------------
// shared-memory matrix descriptor (tcgen05 form, version 1).
// layout 0, no swizzle: 8 x 16-byte core matrices; LBO = byte distance
//   between core matrices adjacent in K, SBO = between those adjacent in M/N.
// layout 1, 128-byte swizzle with 32-byte atoms (the form M-major TF32
//   operands need): atoms of 128 bytes along M/N x 4 K rows; LBO = distance
//   between atoms adjacent in M/N, SBO = between groups of 4 K.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout = 0) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // version 1 (sm_100)
  d |= (uint64_t)(layout & 7u) << 61;
  // base offset 0 (atoms start on their pattern's alignment), leading-offset mode 0
  return d;
}

// instruction descriptor of kind::tf32 / kind::f16 (BF16 inputs): FP32
// accumulator, both operands K-major (a_major = b_major = 0) or MN-major
// (1), M = 128, N a multiple of 16 in [16, 256]
__host__ __device__ constexpr uint32_t idesc(int ab_format, int n, int a_mn_major, int b_mn_major) {
  return (1u << 4)                              // D format F32
         | ((uint32_t)ab_format << 7)            // A format (TF32 = 2, BF16 = 1)
         | ((uint32_t)ab_format << 10)           // B format
         | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
         ((uint32_t)(n >> 3) << 17)               // N >> 3
         | ((uint32_t)(128 >> 4) << 24);          // M >> 4
}
constexpr int FMT_BF16 = 1, FMT_TF32 = 2;

template <int KIND>   // 0: tf32, 1: f16 (bf16 inputs)
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc_v,
                                    uint32_t accumulate) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc_v), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc_v), "r"(accumulate)
        : "memory");
  }
}

// The same MMA with A read from tensor memory: a_tmem addresses lane 0 and the
// first column of a 128-lane A tile (row i of A in lane i, K along the
// columns: one TF32 value or two packed BF16 values per 32-bit column).
template <int KIND>
__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc_v,
                                       uint32_t accumulate) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc_v), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc_v), "r"(accumulate)
        : "memory");
  }
}

// arrive once on `bar` when every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one whole warp; the address is written to *dst (smem)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets row
// (lane base + t), columns [col, col + 16)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// the converse: thread t of the warp writes 16 consecutive 32-bit columns of
// lane (lane base + t); tmem_wait_st waits until this thread's stores landed
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------
// operand splits for near-FP32 products on TF32 / BF16 tensor cores
// (Ootomo & Yokota 2022, "Recovering single precision accuracy from Tensor
// Cores"): x = hi + lo with hi = x rounded to nearest in the narrow format
// (low mantissa bits zero), lo = x - hi (exact in FP32) rounded the same way.
// Both parts are exact values of the narrow format, so the tensor core's own
// input conversion leaves them unchanged.
//
// The rounding is Veltkamp's splitting (Dekker 1971; Boldo 2006 shows the
// high part is a rounding to nearest): with t = (2^(24-SIG) + 1) x in FP32,
// hi = t - (t - x) has at most SIG significant bits.  Three full-rate FP32
// operations instead of a conversion instruction, which issues on the
// quarter-rate XU pipe and was the limit of the operand converters.  The
// operations are written as intrinsics so that no FMA contraction changes
// them.  Past |x| = 2^100 (where t could overflow) the mantissa is rounded
// on its bits; NaN stays NaN.
// ---------------------------------------------------------------------------
template <int SIG>
__device__ __forceinline__ float round_sig(float x) {
  constexpr float SIGMA = (float)((1u << (24 - SIG)) + 1u);
  constexpr uint32_t half = 1u << (23 - SIG), mask = ~((1u << (24 - SIG)) - 1u);
  const float t = __fmul_rn(x, SIGMA);
  const float v = __fsub_rn(t, __fsub_rn(t, x));
  const uint32_t b = __float_as_uint(x);
  const float r = x == x ? __uint_as_float((b + half) & mask) : __uint_as_float(b | 0x00400000u);
  return fabsf(x) <= 0x1p100f ? v : r;      // selects, no branch
}
__device__ __forceinline__ float tf32_rn(float x) { return round_sig<11>(x); }
__device__ __forceinline__ float bf16_rn(float x) { return round_sig<8>(x); }

// The split x = hi + lo of N values (hi to SIG bits, lo = x - hi rounded to
// SIG bits), as 32-bit patterns.  The bound |x| <= 2^100 is checked once for
// all N values; below it the three-operation form alone runs (NaN stays NaN).
template <int SIG>
__device__ __forceinline__ float veltkamp_hi(float x) {
  constexpr float SIGMA = (float)((1u << (24 - SIG)) + 1u);
  const float t = __fmul_rn(x, SIGMA);
  return __fsub_rn(t, __fsub_rn(t, x));
}
// The split of values known to be finite and at most 2^100 in magnitude
// (the factor pool, checked when a plan is built): rounding to SIG bits on
// the bit pattern (add half a unit of the last kept bit, clear the rest:
// round to nearest, ties away from zero; a carry into the exponent is the
// correct rounding up), lo = x - hi exact in FP32 and rounded the same way.
// Two integer operations per rounding instead of three FP32 operations.
// (Packed FP32x2 arithmetic does not serve here: the assembler contracts the
// Veltkamp sequence into fused operations, which returns hi = x.)
template <int SIG, int N>
__device__ __forceinline__ void split_fast(const float (&x)[N], uint32_t (&hi)[N], uint32_t (&lo)[N]) {
  constexpr uint32_t half = 1u << (23 - SIG), mask = ~((1u << (24 - SIG)) - 1u);
#pragma unroll
  for (int e = 0; e < N; ++e) {
    const uint32_t h = (__float_as_uint(x[e]) + half) & mask;
    const float d = __fsub_rn(x[e], __uint_as_float(h));
    hi[e] = h;
    lo[e] = (__float_as_uint(d) + half) & mask;
  }
}
template <int SIG, int N>
__device__ __forceinline__ void split_n(const float (&x)[N], uint32_t (&hi)[N], uint32_t (&lo)[N]) {
  float mx = 0.f;
#pragma unroll
  for (int e = 0; e < N; ++e) mx = fmaxf(mx, fabsf(x[e]));
  if (mx <= 0x1p100f) {
#pragma unroll
    for (int e = 0; e < N; ++e) {
      const float h = veltkamp_hi<SIG>(x[e]);
      hi[e] = __float_as_uint(h);
      lo[e] = __float_as_uint(veltkamp_hi<SIG>(__fsub_rn(x[e], h)));
    }
  } else {
#pragma unroll
    for (int e = 0; e < N; ++e) {
      const float h = round_sig<SIG>(x[e]);
      hi[e] = __float_as_uint(h);
      lo[e] = __float_as_uint(round_sig<SIG>(__fsub_rn(x[e], h)));
    }
  }
}

}  // namespace tc
}  // namespace hm
