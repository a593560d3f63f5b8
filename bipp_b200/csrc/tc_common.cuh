// Helpers for 5th-generation tensor-core kernels (sm_100a): shared-memory matrix
// descriptors, tcgen05.mma (kind::tf32) issue and commit, bounded mbarrier waits, the
// 3xTF32 operand split and tensor-memory loads.
#pragma once

#include <cstdint>

namespace bippb200 {

// spin limit of one wait on the MMA barrier (each try_wait suspends for a bounded time)
constexpr int kTcSpin = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, canonical K-major layout without swizzle: 8-row core
// matrices of 16 bytes per row (128 B contiguous), `sbo` between 8-row groups, `lbo`
// between the two 16-byte K halves of a K-step; version 1 (sm_100)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// the same MMA with the A operand in tensor memory (M = 128: lane i holds row i, one
// 32-bit column per tf32 element along K)
__device__ __forceinline__ void tc_mma_ta(uint32_t dtmem, uint32_t atmem, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// this thread's lane, 8 consecutive 32-bit columns from taddr (warp w may address lanes
// 32 w .. 32 w + 31 only)
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
               "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
               "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
               : "memory");
}

// this thread's tensor-memory stores complete
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// suspend-time hint of one try (ns): a waiting thread is suspended until the phase
// completes or this time passes, instead of spinning and taking issue slots from the
// other warps of the SM
constexpr uint32_t kTcWaitHintNs = 1000;

// bounded wait (at most `spins` tries) for the completion of phase `parity` of the barrier
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int spins = kTcSpin) {
  for (int i = 0; i < spins; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity), "n"(kTcWaitHintNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

// x = hi + lo with hi rounded to the 11 significant bits of tf32 (integer rounding of
// the bit pattern, no conversion instruction) and lo = x - hi exact (|lo| <= 2^-11 |x|);
// the tensor core reads lo's top 11 bits, so the split keeps ~22 significant bits
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
  hi = __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
  lo = x - hi;
}

// split_tf32 of two values; lo = hi * (-1) + x exactly, one packed FMA for both
__device__ __forceinline__ void split_tf32x2(float2 x, float2& hi, float2& lo) {
  hi.x = __uint_as_float((__float_as_uint(x.x) + 0x1000u) & 0xFFFFE000u);
  hi.y = __uint_as_float((__float_as_uint(x.y) + 0x1000u) & 0xFFFFE000u);
  lo = __ffma2_rn(hi, make_float2(-1.f, -1.f), x);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, float a, float b, float c, float d) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
  uint32_t u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
        "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}

}  // namespace bippb200
