// tcgen05 (5th-generation tensor core) helpers shared by the tensor-core
// kernels: the no-swizzle K-major shared-memory operand layout, its UMMA
// descriptor, the 16-bit instruction descriptor, MMA issue/commit and TMEM
// loads.  One thread issues the MMAs of a CTA; accumulators live in TMEM.
#pragma once

#include <cuda_runtime.h>

#include "device_util.cuh"

namespace ksvd {

// Byte offset of element (r, k) of an R x Kd BF16 K-major operand in the
// no-swizzle canonical layout: core matrix (k/8, r/8) of 8 rows x 16 bytes.
__device__ __forceinline__ unsigned canon_off(int r, int k, int R) {
  return unsigned(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// UMMA shared-memory descriptor: no swizzle, K-major; LBO = byte distance of
// K-adjacent core matrices, SBO = byte distance of row-adjacent ones.
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  unsigned long long d = 0;
  d |= (unsigned long long)((saddr >> 4) & 0x3FFFu);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version for sm_100
  return d;          // base offset 0, LBO mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor: 16-bit x 16-bit -> FP32 (fmt: 0 = F16, 1 = BF16),
// A and B K-major, M x N.
__host__ __device__ constexpr unsigned umma_idesc_16(int M, int N, unsigned fmt) {
  return (1u << 4)                       // D format F32
         | (fmt << 7)                    // A format
         | (fmt << 10)                   // B format
         | (unsigned(N >> 3) << 17)      // N / 8
         | (unsigned(M >> 4) << 24);     // M / 16
}

KSVD_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
KSVD_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

KSVD_DEV void tc_mma(unsigned d_tmem, unsigned long long adesc, unsigned long long bdesc, unsigned idesc,
                     unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

KSVD_DEV void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
KSVD_DEV void tc_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
KSVD_DEV void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
KSVD_DEV void tc_ld32(unsigned taddr, float (&v)[32]) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}


// 8 consecutive FP32 columns of this thread's TMEM lane.
KSVD_DEV void tc_ld8(unsigned taddr, float (&v)[8]) {
  unsigned r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

KSVD_DEV void tc_alloc(unsigned* slot_smem, unsigned cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

KSVD_DEV void tc_dealloc(unsigned tmem, unsigned cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

}  // namespace ksvd
