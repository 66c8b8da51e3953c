// tc_common.cuh -- fifth-generation tensor core (tcgen05) building blocks for
// sm_100a: TMEM allocation, shared-memory matrix descriptors, BF16 MMA with
// FP32 accumulation in TMEM, commit to an mbarrier, bounded waits, TMEM loads.
//
// Operand layout used throughout (K-major, no swizzle): a tile of R rows by
// KD bf16 columns (KD a multiple of 16) is stored as 8x8 "core matrices" of
// 128 contiguous bytes; element (r, k) lives at byte
//     ((r / 8) * (KD / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// For the MMA step covering k in [16 s, 16 s + 16) the descriptor starts at
// byte 256 s, the two 8-column core matrices along K are 128 bytes apart
// (leading byte offset) and consecutive 8-row groups KD * 16 bytes apart
// (stride byte offset).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace knnsweet {
namespace tc {

// Bytes of one R x KD tile in the core-matrix layout.
__host__ __device__ constexpr size_t tile_bytes(int rows, int kd) {
  return (size_t)rows * kd * 2;
}

// Byte offset of element (r, k) inside a tile with KD columns.
__host__ __device__ __forceinline__ uint32_t tile_offset(int r, int k, int kd) {
  return (uint32_t)((((r >> 3) * (kd >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16 (both K-major), D = F32.
__host__ __device__ constexpr uint32_t make_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

// TMEM allocation of `ncols` columns (power of two >= 32) by one full warp;
// the base address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_u32(dst)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
               :: "r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T for one K = 16 step.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// Arrive on the mbarrier once every tcgen05 operation issued so far by this
// thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's generic-proxy shared-memory writes visible to the
// tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count)
               : "memory");
}

// One arrival on the mbarrier that also expects `bytes` of asynchronous
// copies to complete in the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// One plain arrival on the mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(mbar)) : "memory");
}

// 1-D bulk asynchronous copy global -> this CTA's shared memory (no
// multicast), completing `bytes` of transaction count on the mbarrier.  Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *dst_smem, const void *src_gmem,
                                              uint32_t bytes, uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(smem_u32(dst_smem)), "l"(src_gmem), "r"(bytes), "r"(smem_u32(mbar))
      : "memory");
}

// Bounded wait for the mbarrier phase with the given parity.  Returns false
// when the wait gives up (about a second of spinning).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t addr = smem_u32(mbar);
  for (uint32_t it = 0; it < (1u << 24); it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

// 32 lanes x 32 columns of 32-bit values: thread t of the warp receives the
// 32 consecutive columns of TMEM lane (lane base + t).  The load and its wait
// are one asm statement, so no use of the registers can be scheduled before
// the data has arrived.
__device__ __forceinline__ void tmem_ld_32x32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
        "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace knnsweet
