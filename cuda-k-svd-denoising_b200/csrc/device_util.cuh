// Device helpers: warp reductions, acquire/release accesses, the bounded
// software grid barrier of the persistent kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "ksvd_internal.cuh"

namespace ksvd {

#define KSVD_DEV __device__ __forceinline__

// Wall-clock limit of one grid-barrier wait (ns).  A wait that runs this long
// sets DEVERR_TIMEOUT and returns; every later wait sees the flag and returns
// at once, so a failed launch ends within about this long.
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;

KSVD_DEV unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

KSVD_DEV unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

KSVD_DEV void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

KSVD_DEV int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T>
KSVD_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

KSVD_DEV float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; `red` is shared scratch of at least 32 elements.  All
// threads get the result.
template <typename T>
__device__ T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  T t = (threadIdx.x < nw) ? red[threadIdx.x] : T(0);
  if (warp == 0) t = warp_sum(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  return red[0];
}

// Block-wide sum of a pair; `red` holds at least 64 floats.
__device__ inline float2 block_sum2(float2 v, float* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  __syncthreads();
  if (lane == 0) {
    red[2 * warp] = v.x;
    red[2 * warp + 1] = v.y;
  }
  __syncthreads();
  float2 t = (threadIdx.x < nw) ? make_float2(red[2 * threadIdx.x], red[2 * threadIdx.x + 1]) : make_float2(0.f, 0.f);
  if (warp == 0) {
    t.x = warp_sum(t.x);
    t.y = warp_sum(t.y);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    red[0] = t.x;
    red[1] = t.y;
  }
  __syncthreads();
  return make_float2(red[0], red[1]);
}

__device__ inline float block_max(float v, float* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  float t = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0f;
  if (warp == 0) t = warp_max(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  return red[0];
}

// Software grid barrier for a cooperative launch (all CTAs co-resident).
// Returns false when an error is flagged: this CTA's wait timed out, or
// another CTA flagged one.  Every wait is bounded by kBarrierTimeoutNs.
__device__ inline bool grid_sync(GridBarrier* b, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned gen = ld_acquire_u32(&b->gen);
    __threadfence();
    unsigned arrived = atomicAdd(&b->count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      st_release_u32(&b->gen, gen + 1u);
    } else {
      unsigned long long t0 = globaltimer_ns();
      while (ld_acquire_u32(&b->gen) == gen) {
        if (ld_relaxed_i32(&b->err) != DEVERR_NONE) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > kBarrierTimeoutNs) {
          atomicCAS(&b->err, DEVERR_NONE, DEVERR_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    if (ok && ld_relaxed_i32(&b->err) != DEVERR_NONE) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// mbarrier + bulk (TMA) copies global -> shared.
// ---------------------------------------------------------------------------
KSVD_DEV unsigned smem_u32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

KSVD_DEV void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

KSVD_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses of the same bytes.
KSVD_DEV void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

KSVD_DEV void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy; dst, src 16-byte aligned, bytes a multiple of 16.
// Hint: bring [src, src + bytes) into L2 (16-byte aligned, a multiple of 16
// bytes, inside an allocation).
KSVD_DEV void bulk_prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

KSVD_DEV void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

KSVD_DEV bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete, at most timeout_ns.
KSVD_DEV bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity))
    if (globaltimer_ns() - t0 > timeout_ns) return false;
  return true;
}

}  // namespace ksvd
