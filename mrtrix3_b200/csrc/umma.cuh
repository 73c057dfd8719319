// sm_100a building blocks shared by the tcgen05 kernels (projection pass,
// warm-start network inference): shared-memory matrix descriptors for the
// canonical K-major, non-swizzled layout (8-row x 16-byte core matrices),
// the kind::f16 instruction descriptor, bounded mbarrier waits, bulk
// global -> shared copies completing on an mbarrier, and the tcgen05
// issue / commit / load / fence wrappers.  Every wait is bounded: callers
// turn a time-out into an error flag instead of spinning forever.
#pragma once

#include <cstdint>

namespace csdb200 {

constexpr unsigned kTcWaitLimit = 1u << 26;

// Shared-memory matrix descriptor: start address, leading byte offset (the
// distance between the two K-adjacent core matrices of one K=16 step) and
// stride byte offset (the distance between 8-row groups), version 1, no
// swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);             // start address, bits [0,14)
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;         // leading (K-chunk) byte offset, bits [16,30)
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;         // stride (row-group) byte offset, bits [32,46)
  d |= (uint64_t)1 << 46;                             // descriptor version 1 (sm_100)
  return d;                                           // base offset 0, no swizzle (layout type 0)
}

// kind::f16 instruction descriptor: F32 D, K-major A and B, both operands
// F16 (bf16 = false) or both BF16 (bf16 = true).
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N, bool bf16 = false) {
  return (1u << 4) | (bf16 ? ((1u << 7) | (1u << 10)) : 0u) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity));
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count));
}

// One arrival that also expects `bytes` of bulk-copy transactions.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}

// Bulk copy (no tensor map, no multicast) of `bytes` (a multiple of 16, both
// addresses 16-byte aligned) from this GPU's global memory into this CTA's
// shared memory; completes as transactions on `mbar`.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(mbar)
      : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one instruction, issued by one thread.
__device__ __forceinline__ void umma_f16_ss(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred q;\n\t"
      "setp.ne.b32 q, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, q;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on `mbar` once every tcgen05.mma this thread issued so far is done.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar));
}

// 16 consecutive 32-bit columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::); }
// make this thread's generic-proxy shared-memory writes visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::); }

// Tensor-memory allocation of `cols` columns by one whole warp; the base
// address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot_saddr), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols));
}

}  // namespace csdb200
