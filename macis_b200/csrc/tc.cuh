// sm_100a tensor-core plumbing in inline PTX: mbarriers with time-bounded
// waits, untiled bulk copies (global -> shared, completion on an mbarrier),
// tcgen05 TMEM allocation, BF16 MMA with FP32 accumulation in TMEM,
// tcgen05.commit and tcgen05.ld.
//
// Operand tiles use the K-major, non-swizzled canonical layout of the
// tcgen05 shared-memory descriptor. A "core matrix" is 8 rows x 16 bytes
// (8 bf16 along K) stored as 128 contiguous bytes. This file stores a tile of
// R rows x K columns as K/8 "slabs", slab s holding column block [8s, 8s+8)
// of all R rows (R x 16 bytes, row r at byte 16 r). Then
//   element (r, k) is at byte (k / 8) * 16 R + 16 r + 2 (k % 8),
//   descriptor SBO (stride between 8-row groups) = 128 bytes,
//   descriptor LBO (stride between the two K core matrices of one K=16 MMA)
//   = 16 R bytes, and the MMA for K columns [16 j, 16 j + 16) starts at slab
//   2 j.
// A thread that owns row r writes its 16-byte pieces at 16 r + s * 16 R, so a
// warp writing 32 consecutive rows of one slab touches 512 contiguous bytes.
#pragma once
#include <cstdint>

namespace mb {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ------------------------------------------------------------- mbarriers
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count)
               : "memory");
}
// Make initialised barriers visible to the async proxy (bulk copies, MMA
// commits) before any thread uses them.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for completion of the phase with the given parity, at most
// `limit_ns` nanoseconds. Returns false on timeout (the caller records the
// error and stops issuing work; nothing here spins without bound).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint64_t limit_ns = 2000000000ull) {
  if(mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while(!mbar_try_wait(bar, parity))
    if(global_ns() - t0 > limit_ns) return false;
  return true;
}

// ------------------------------------------------------------ bulk copy
// Untiled bulk copy global -> shared; both addresses 16-byte aligned and
// `bytes` a multiple of 16. Completion is reported on `bar` (transaction
// bytes), which the caller armed with mbar_expect_tx.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src,
                                         uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Generic-proxy shared-memory writes -> visible to tcgen05.mma / bulk copies.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ------------------------------------------------------------------ TMEM
// Whole-warp calls. `ncols` is a power of two >= 32.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile(
      "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
          smem_addr(slot)),
      "r"(ncols)
      : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::
                   : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                   taddr),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ------------------------------------------------------------ descriptors
// Shared-memory matrix descriptor, non-swizzled K-major (version 1 = sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo,
                                          uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFF);
  d |= uint64_t((lbo >> 4) & 0x3FFF) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;  // version
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}
// Instruction descriptor, kind::f16: A = B = BF16, D = F32, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4)                      // D format F32
         | (1u << 7)                    // A format BF16
         | (1u << 10)                   // B format BF16
         | (uint32_t(N >> 3) << 17)     // N / 8
         | (uint32_t(M >> 4) << 24);    // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da,
                                         uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive once on `bar` when every MMA this thread issued so far completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
      "[%0];" ::"r"(smem_addr(bar))
      : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns; thread t of the warp gets lane
// (lane base + t). `taddr` = (lane base << 16) | column.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]),
        "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
        "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
        "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc
}  // namespace mb
