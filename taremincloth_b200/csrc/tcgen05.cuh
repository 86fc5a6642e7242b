// Fifth-generation tensor core (tcgen05) building blocks for sm_100a:
// shared-memory matrix descriptors, the kind::f16 instruction descriptor,
// tensor-memory (TMEM) allocation, MMA issue, completion through an
// mbarrier with a bounded wait, and TMEM loads for the epilogue.
//
// Operand layout used here (K-major, no swizzle): the matrix is cut into
// core matrices of 8 rows x 16 bytes (8 bf16 along K), each stored as 128
// contiguous bytes, row r of the core matrix at byte 16 r.  With K_total
// elements per row, core matrix (row group g, K chunk c) sits at byte
// (g * K_total / 8 + c) * 128, so one MMA step of K = 16 reads chunks 2s and
// 2s + 1: leading byte offset (next chunk along K) = 128, stride byte offset
// (next 8-row group) = K_total / 8 * 128, start address + 256 s.
#pragma once
#include <cstdint>

namespace tcloth {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, k) in the core-matrix layout above.
__device__ __forceinline__ uint32_t cm_offset(uint32_t row, uint32_t k, uint32_t k_total) {
  return ((row >> 3) * (k_total >> 3) + (k >> 3)) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// and stride byte offsets in 16-byte units, version 1 at bits 46-47, base
// offset 0, layout type 0 (no swizzle) at bits 61-63.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: D f32 (bits 4-5 = 1),
// A and B bf16 (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0),
// N / 8 at bits 17-22, M / 16 at bits 24-28, dense, no negation.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t m, uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole
// warp; the base address is written to shared memory at `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, one elected thread, cta_group::1.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}
// Arrive on the mbarrier once every MMA this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}
// Waits for the phase with parity `parity` to complete, polling at most
// `limit` times with a short sleep in between; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_addr(mbar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(64);
  }
  return false;
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (32x32b shape:
// warp w of the CTA reads lanes 32 (w % 4) .. 32 (w % 4) + 31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  // the registers are read-write operands of the wait, so no use of them
  // can be scheduled before it
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tcloth
