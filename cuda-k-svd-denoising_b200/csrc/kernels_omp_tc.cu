// Batched OMP with the correlation D^T R on the 5th-generation tensor cores
// (CuBlasMatrixOmp::work, cublas_matrix_omp.cu:107-402, BF16 form).
//
// Per CTA (persistent over tiles of 128 patches, one CTA per SM):
//   * the dictionary lives in shared memory as the BF16 B operand (atoms x n,
//     K-major, no swizzle: 8-row x 16-byte core matrices);
//   * each OMP step, one thread issues n/16 tcgen05.mma (M = 128 patches,
//     N = atoms, K = 16, BF16 inputs, FP32 accumulation in tensor memory) and
//     commits them to an mbarrier;
//   * thread m of the 128 epilogue threads owns TMEM lane m = patch m: it
//     streams its row of correlations out of tensor memory (tcgen05.ld),
//     keeps the kTopT largest |c|, re-scores those candidates exactly,
//         c_a = d_a . y - sum_s g_s <d_a, d_s>   (FP64, FP32 inputs)
//     and takes the largest, lowest atom index on ties (cublasIsamax,
//     :216-233);
//   * it extends the Cholesky factor of its support Gram (FP64, from the FP64
//     dictionary Gram), solves for the coefficients (the reference's
//     pseudo-inverse, :269-339), forms the FP32 residual y - D_S g and its
//     norm (:352-393; stop when below 1e-3, :218) and writes the residual as
//     BF16 into the A operand of the next step.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kTcTile = 128;     // patches per tile = UMMA M = TMEM lanes
constexpr int kTcThreads = 128;  // one epilogue thread per patch
constexpr int kTopT = 8;         // BF16 candidates re-scored exactly
constexpr int kTcLMax = 16;
constexpr unsigned long long kMmaWaitNs = 2000000000ull;

struct TcLayout {
  int Kp, np16, ysn, tri;
  size_t off_b, off_a, off_y, off_lc, off_bv, off_s, off_gam, off_bar, off_tmem, total;
  unsigned tmem_cols;
};

__host__ __device__ inline size_t tc_al(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline TcLayout tc_layout(int n, int K, int L) {
  TcLayout o;
  o.Kp = int(tc_al(K, 16));
  o.np16 = int(tc_al(n, 16));
  o.ysn = n + 1;
  o.tri = L * (L + 1) / 2;
  size_t off = 0;
  o.off_b = off;
  off = tc_al(off + size_t(o.Kp) * o.np16 * 2, 128);
  o.off_a = off;
  off = tc_al(off + size_t(kTcTile) * o.np16 * 2, 128);
  o.off_y = off;
  off = tc_al(off + size_t(kTcTile) * o.ysn * 4, 16);
  o.off_lc = off;
  off = tc_al(off + size_t(kTcTile) * o.tri * 8, 16);
  o.off_bv = off;
  off = tc_al(off + size_t(kTcTile) * L * 8, 16);
  o.off_s = off;
  off = tc_al(off + size_t(kTcTile) * L * 4, 16);
  o.off_gam = off;
  off = tc_al(off + size_t(kTcTile) * L * 4, 16);
  o.off_bar = off;
  off = tc_al(off + 16, 16);
  o.off_tmem = off;
  off = tc_al(off + 16, 16);
  o.total = off;
  unsigned cols = 32;
  while (cols < unsigned(o.Kp)) cols <<= 1;
  o.tmem_cols = cols;
  return o;
}

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

// Instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M x N.
__host__ __device__ constexpr unsigned umma_idesc_bf16(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
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

__global__ void __launch_bounds__(kTcThreads, 1)
    omp_tc_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                  const double* __restrict__ Gram, int K, int L, int32_t* __restrict__ idx_out,
                  float* __restrict__ coef_out, int64_t ntiles, int d_vec4, GridBarrier* flags, DevStats* stats) {
  extern __shared__ __align__(128) unsigned char smem[];
  const TcLayout lo = tc_layout(n, K, L);
  unsigned char* Bt = smem + lo.off_b;
  unsigned char* At = smem + lo.off_a;
  float* Ys = reinterpret_cast<float*>(smem + lo.off_y);
  double* Lc = reinterpret_cast<double*>(smem + lo.off_lc);
  double* bv = reinterpret_cast<double*>(smem + lo.off_bv);
  int* Ss = reinterpret_cast<int*>(smem + lo.off_s);
  float* gam = reinterpret_cast<float*>(smem + lo.off_gam);
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(smem + lo.off_bar);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(smem + lo.off_tmem);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int Kp = lo.Kp, np16 = lo.np16, ysn = lo.ysn, tri = lo.tri;

  // ---- set-up: TMEM, mbarrier, BF16 dictionary operand ---------------------
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(lo.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(mbar, 1);
    fence_mbar_init();
  }
  for (int t = tid; t < Kp * (np16 / 8); t += kTcThreads) {
    const int a = t / (np16 / 8), kc = t - a * (np16 / 8);
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int k = kc * 8 + e;
      h[e] = __float2bfloat16_rn((a < K && k < n) ? __ldg(D + int64_t(a) * n + k) : 0.0f);
    }
    *reinterpret_cast<uint4*>(Bt + canon_off(a, kc * 8, Kp)) = *reinterpret_cast<const uint4*>(h);
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned idesc = umma_idesc_bf16(kTcTile, Kp);
  const unsigned a_base = smem_u32(At), b_base = smem_u32(Bt);
  unsigned phase = 0;
  bool failed = false;

  const int m = tid;  // this thread's patch (and TMEM lane) within a tile
  const unsigned lane_addr = tmem + (unsigned(warp * 32) << 16);

  for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const int64_t p0 = tile * kTcTile;
    const int np = (N - p0 < kTcTile) ? int(N - p0) : kTcTile;
    // patch tile: FP32 copy (odd row stride) and the BF16 A operand
    for (int t = tid; t < kTcTile * n; t += kTcThreads) {
      const int p = t / n, k = t - p * n;
      Ys[p * ysn + k] = (p < np) ? __ldg(Y + p0 * n + t) : 0.0f;
    }
    __syncthreads();
    int cnt = 0;
    bool done = m >= np;
    {
      const float* yr = Ys + m * ysn;
      for (int kc = 0; kc < np16 / 8; ++kc) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = kc * 8 + e;
          h[e] = __float2bfloat16_rn(k < n ? yr[k] : 0.0f);
        }
        *reinterpret_cast<uint4*>(At + canon_off(m, kc * 8, kTcTile)) = *reinterpret_cast<const uint4*>(h);
      }
    }
    for (int step = 0; step < L; ++step) {
      fence_proxy_async_smem();
      tc_fence_before();
      if (!__syncthreads_or(!done)) break;
      // ---- correlation on the tensor cores ---------------------------------
      if (tid == 0) {
        tc_fence_after();
        for (int kk = 0; kk < np16 / 16; ++kk) {
          const unsigned long long ad = umma_desc(a_base + kk * 2 * kTcTile * 16, kTcTile * 16, 128);
          const unsigned long long bd = umma_desc(b_base + kk * 2 * Kp * 16, Kp * 16, 128);
          tc_mma(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc_commit(mbar);
      }
      const bool ok = mbar_wait(mbar, phase, kMmaWaitNs);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicCAS(&flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
        failed = true;
        phase ^= 1u;  // the drain waits for the phase that did not complete
        break;
      }
      tc_fence_after();
      // ---- top-T candidates by |BF16 correlation| --------------------------
      float tv[kTopT];
      int ta[kTopT];
#pragma unroll
      for (int q = 0; q < kTopT; ++q) {
        tv[q] = -1.0f;
        ta[q] = -1;
      }
      for (int c0 = 0; c0 < Kp; c0 += 32) {
        float v[32];
        tc_ld32(lane_addr + unsigned(c0), v);  // warp-collective: all lanes load
        if (!done) {
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const int a = c0 + i;
            const float av = fabsf(v[i]);
            if (a < K && av > tv[kTopT - 1]) {
              int q = kTopT - 1;
              while (q > 0 && av > tv[q - 1]) {
                tv[q] = tv[q - 1];
                ta[q] = ta[q - 1];
                --q;
              }
              tv[q] = av;
              ta[q] = a;
            }
          }
        }
      }
      if (!done) {
        // ---- exact re-score: c_a = d_a.y - sum_s g_s G[a][s] ----------------
        const float* yr = Ys + m * ysn;
        double best = -1.0, best_b = 0.0;
        int best_a = -1;
        for (int q = 0; q < kTopT; ++q) {
          const int a = ta[q];
          if (a < 0) continue;
          const float4* dr = reinterpret_cast<const float4*>(D + int64_t(a) * n);
          double ba = 0.0;
          if (d_vec4) {
            for (int k4 = 0; k4 < n / 4; ++k4) {
              const float4 d4 = __ldg(dr + k4);
              ba = fma(double(d4.x), double(yr[4 * k4]), ba);
              ba = fma(double(d4.y), double(yr[4 * k4 + 1]), ba);
              ba = fma(double(d4.z), double(yr[4 * k4 + 2]), ba);
              ba = fma(double(d4.w), double(yr[4 * k4 + 3]), ba);
            }
          } else {
            for (int k = 0; k < n; ++k) ba = fma(double(__ldg(D + int64_t(a) * n + k)), double(yr[k]), ba);
          }
          double ca = ba;
          for (int s = 0; s < cnt; ++s) ca -= double(gam[m * L + s]) * Gram[int64_t(a) * K + Ss[m * L + s]];
          const double aca = fabs(ca);
          if (aca > best || (aca == best && a < best_a)) {
            best = aca;
            best_a = a;
            best_b = ba;
          }
        }
        const int a = best_a < 0 ? 0 : best_a;
        bool stop = false;
        for (int s = 0; s < cnt; ++s)
          if (Ss[m * L + s] == a) stop = true;  // re-selected atom: the pursuit ends
        if (!stop) {
          // ---- Cholesky row append (packed lower triangle) and solve --------
          double* Lp = Lc + m * tri;
          auto Lat = [&](int i, int j) -> double& { return Lp[i * (i + 1) / 2 + j]; };
          const int k = cnt;
          double ww = 0.0;
          for (int i = 0; i < k; ++i) {
            double s = Gram[int64_t(Ss[m * L + i]) * K + a];
            for (int j = 0; j < i; ++j) s -= Lat(i, j) * Lat(k, j);
            const double wi = s / Lat(i, i);
            Lat(k, i) = wi;
            ww += wi * wi;
          }
          const double piv2 = Gram[int64_t(a) * K + a] - ww;
          if (!(piv2 > 0.0)) {
            stop = true;
          } else {
            Lat(k, k) = sqrt(piv2);
            Ss[m * L + k] = a;
            bv[m * L + k] = best_b;
            cnt = k + 1;
            double yv[kTcLMax];
            for (int i = 0; i <= k; ++i) {
              double s = bv[m * L + i];
              for (int j = 0; j < i; ++j) s -= Lat(i, j) * yv[j];
              yv[i] = s / Lat(i, i);
            }
            for (int i = k; i >= 0; --i) {
              double s = yv[i];
              for (int j = i + 1; j <= k; ++j) s -= Lat(j, i) * yv[j];
              yv[i] = s / Lat(i, i);
            }
            for (int i = 0; i <= k; ++i) gam[m * L + i] = float(yv[i]);
          }
        }
        if (stop) {
          done = true;
        } else {
          // ---- residual (FP32), its norm, and the next A operand ------------
          float nrm = 0.0f;
          for (int kc = 0; kc < np16 / 8; ++kc) {
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int kk = kc * 8 + e;
              float r = 0.0f;
              if (kk < n) {
                r = yr[kk];
                for (int s = 0; s < cnt; ++s) r = fmaf(-gam[m * L + s], __ldg(D + int64_t(Ss[m * L + s]) * n + kk), r);
                nrm = fmaf(r, r, nrm);
              }
              h[e] = __float2bfloat16_rn(r);
            }
            *reinterpret_cast<uint4*>(At + canon_off(m, kc * 8, kTcTile)) = *reinterpret_cast<const uint4*>(h);
          }
          if (sqrtf(nrm) < 1e-3f) done = true;
        }
      }
    }
    // ---- compact codes ------------------------------------------------------
    if (m < np) {
      for (int s = 0; s < L; ++s) {
        const bool used = s < cnt;
        idx_out[(p0 + m) * L + s] = used ? Ss[m * L + s] : -1;
        coef_out[(p0 + m) * L + s] = used ? gam[m * L + s] : 0.0f;
      }
    }
    __syncthreads();
  }
  // ---- teardown --------------------------------------------------------------
  if (failed && tid == 0) mbar_wait(mbar, phase, kMmaWaitNs);  // bounded drain of MMAs in flight
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(lo.tmem_cols) : "memory");
  }
  (void)stats;
}

size_t omp_tc_smem_bytes(int n, int K, int L) { return tc_layout(n, K, L).total; }

bool omp_tc_supported(int n, int K, int L) {
  return L >= 1 && L <= kTcLMax && n >= 1 && K >= 1 && tc_al(K, 16) <= 256 && omp_tc_smem_bytes(n, K, L) <= 227 * 1024;
}

cudaError_t launch_omp_tc(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K, int L,
                          int32_t* idx, float* coef, int num_sms, GridBarrier* flags, DevStats* stats,
                          cudaStream_t s) {
  const size_t smem = omp_tc_smem_bytes(n, K, L);
  cudaError_t e = cudaFuncSetAttribute(omp_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int64_t ntiles = (N + kTcTile - 1) / kTcTile;
  const int grid = int(std::min<int64_t>(ntiles, num_sms));
  const int d_vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(dict) & 15) == 0) ? 1 : 0;
  omp_tc_kernel<<<grid, kTcThreads, smem, s>>>(patches, N, n, dict, gram, K, L, idx, coef, ntiles, d_vec4, flags,
                                               stats);
  return cudaGetLastError();
}

}  // namespace ksvd
