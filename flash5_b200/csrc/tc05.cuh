// tc05.cuh -- the sm_100a tensor-core primitives of the batched network
// inference (riemann_exact.cu): tensor memory (TMEM) allocation,
// shared-memory matrix descriptors, tcgen05.mma of kind f16 issued by one
// thread, its completion through tcgen05.commit on an mbarrier, and
// tcgen05.ld of the FP32 accumulators back to registers.
//
// Operand layout: the canonical K-major layout without swizzle.  A matrix
// of R rows and K BF16 columns is stored as core matrices of 8 rows x 16
// bytes (8 values along K), each core matrix 128 contiguous bytes; core
// matrices adjacent along K are LBO = 128 bytes apart and groups of 8 rows
// are SBO = K/8 * 128 bytes apart.  One MMA of kind f16 consumes K = 16
// (two core matrices along K); the next K-step starts 256 bytes further.
// The accumulator of an M = 128 MMA with cta_group::1 holds row m in TMEM
// lane m, column n in TMEM column n (FP32), so warp w of a 128-thread CTA
// reads rows 32w..32w+31, one row per lane.
#pragma once
#include <stdint.h>

namespace tc05 {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of (row, 16-byte chunk along K) in the canonical layout
__host__ __device__ constexpr uint32_t canon_off(int row, int chunk, uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)chunk * 128u + (uint32_t)(row & 7) * 16u;
}

// shared-memory matrix descriptor (sm_100): start address >> 4 in bits
// 0-13, LBO >> 4 in 16-29, SBO >> 4 in 32-45, descriptor version 1 in
// 46-47, base offset 0, layout type 0 (no swizzle) in 61-63
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor of kind f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in
// bits 17-22, M >> 4 in bits 24-28
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_bf16_f32() {
  static_assert(M == 128 && N % 16 == 0 && N >= 16 && N <= 256, "M = 128, N a multiple of 16 up to 256");
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// TMEM columns: a power of two >= 32, allocated and freed by one whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// an mbarrier of `count` arrivals, and one poll of the phase with `parity`
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// polls for at most `cycles` SM clocks; false if the phase did not complete
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, long long cycles) {
  const long long t0 = clock64();
  bool done = mbar_try(bar, parity);
  while (!done && clock64() - t0 < cycles) done = mbar_try(bar, parity);
  return done;
}

// ordering of tcgen05 operations around thread synchronisation
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// generic-proxy shared-memory writes made visible to the tensor cores
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// the mbarrier gets one arrival once every MMA this thread issued before
// has completed
__device__ __forceinline__ void commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 lanes (one row per lane),
// waited for in the same statement so no use of r precedes the wait
__device__ __forceinline__ void ld32(uint32_t taddr, uint32_t r[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

// 2 consecutive FP32 columns of this warp's 32 lanes
__device__ __forceinline__ void ld2(uint32_t taddr, uint32_t r[2]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1])
      : "r"(taddr)
      : "memory");
}

}  // namespace tc05
