// Batched OMP sparse coding, plain FP32 form, for dictionaries too large to
// keep in shared memory (CuBlasMatrixOmp::work, cublas_matrix_omp.cu:107-402).
//
// Same arithmetic, in the same order, as the resident-dictionary kernel in
// kernels_omp.cu, so both give identical codes where both apply; only the
// data movement differs.  Per tile of kSP patches and per OMP step the
// dictionary streams through shared memory in chunks of KC features that
// span all atoms (k-major).  While a chunk is resident the CTA
//   1. forms the chunk's rows of the residual y - D_S g of the previous
//      step's least squares (:352-380), with their contribution to its norm,
//   2. accumulates the chunk's part of the correlation D^T r (register tiles
//      of APT atoms x 4 patches per thread).
// After the last chunk, patches whose residual norm fell below 1e-3 stop
// (:218) and the others take the argmax |.| with the lowest atom index on
// ties (cublasIsamax, :216-233), then the Cholesky least squares of the
// resident kernel (FP64, support Gram from the FP64 dictionary Gram).
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kSP = 32;          // patches per tile
constexpr int kSThreads = 256;   // 32 atom groups x 8 patch groups
constexpr int kSLMax = 32;
constexpr size_t kSSmemMax = 227 * 1024 - 256;

struct OmpSLayout {
  int Kpad, dks, rks, ysn, KC;
  size_t off_dk, off_rk, off_ys, off_lc, off_bv, off_s, off_gam, off_sel, off_cnt, off_done, off_redv, off_redi,
      off_gs, off_bs, off_np, total;
};

__host__ __device__ inline size_t s_al16(size_t x) { return (x + 15) & ~size_t(15); }

// Kpad = 32 * apt atoms; KC features per dictionary chunk (0: does not fit).
__host__ __device__ inline OmpSLayout omp_s_layout(int n, int apt, int L) {
  OmpSLayout o;
  o.Kpad = 32 * apt;
  o.dks = o.Kpad + 4;
  o.rks = kSP + 4;
  o.ysn = n + 1;
  size_t off = 0;
  o.off_rk = off;
  off = s_al16(off + size_t(n) * o.rks * 4);
  o.off_ys = off;
  off = s_al16(off + size_t(kSP) * o.ysn * 4);
  o.off_lc = off;
  off = s_al16(off + size_t(kSP) * L * L * 8);
  o.off_bv = off;
  off = s_al16(off + size_t(kSP) * L * 8);
  o.off_s = off;
  off = s_al16(off + size_t(kSP) * L * 4);
  o.off_gam = off;
  off = s_al16(off + size_t(kSP) * L * 4);
  o.off_sel = off;
  off = s_al16(off + kSP * 4);
  o.off_cnt = off;
  off = s_al16(off + kSP * 4);
  o.off_done = off;
  off = s_al16(off + kSP * 4);
  o.off_redv = off;
  off = s_al16(off + 8 * kSP * 4);
  o.off_redi = off;
  off = s_al16(off + 8 * kSP * 4);
  o.off_gs = off;
  off = s_al16(off + size_t(kSP) * (L + 1) * 8);
  o.off_bs = off;
  off = s_al16(off + kSP * 8);
  o.off_np = off;
  off = s_al16(off + 8 * kSP * 4);
  o.off_dk = off;
  // the largest chunk (a multiple of 4 features, at most n rounded up) that fits
  const size_t per_k = size_t(o.dks) * 4;
  int kc = 0;
  if (off < kSSmemMax) kc = int((kSSmemMax - off) / per_k) & ~3;
  const int n4 = (n + 3) & ~3;
  if (kc > n4) kc = n4;
  o.KC = kc;
  o.total = off + size_t(kc) * per_k;
  return o;
}

__device__ __forceinline__ bool s_better(float v1, int i1, float v2, int i2) {
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

template <int APT>
__global__ void __launch_bounds__(kSThreads, 1)
    omp_stream_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                      const double* __restrict__ Gram, int K, int L, int32_t* __restrict__ idx_out,
                      float* __restrict__ coef_out, int64_t ntiles, DevStats* stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const OmpSLayout lo = omp_s_layout(n, APT, L);
  float* Dk = reinterpret_cast<float*>(smem + lo.off_dk);
  float* Rk = reinterpret_cast<float*>(smem + lo.off_rk);
  float* Ys = reinterpret_cast<float*>(smem + lo.off_ys);
  double* Lc = reinterpret_cast<double*>(smem + lo.off_lc);
  double* bvec = reinterpret_cast<double*>(smem + lo.off_bv);
  int* S = reinterpret_cast<int*>(smem + lo.off_s);
  float* gam = reinterpret_cast<float*>(smem + lo.off_gam);
  int* sel = reinterpret_cast<int*>(smem + lo.off_sel);
  int* cnt = reinterpret_cast<int*>(smem + lo.off_cnt);
  int* done = reinterpret_cast<int*>(smem + lo.off_done);
  float* redv = reinterpret_cast<float*>(smem + lo.off_redv);
  int* redi = reinterpret_cast<int*>(smem + lo.off_redi);
  double* gS = reinterpret_cast<double*>(smem + lo.off_gs);
  double* bS = reinterpret_cast<double*>(smem + lo.off_bs);
  float* npart = reinterpret_cast<float*>(smem + lo.off_np);
  const int ysn = lo.ysn, dks = lo.dks, rks = lo.rks, Kpad = lo.Kpad, KC = lo.KC;
  // chunks start at multiples of 4 features; rows are 16-byte aligned when n is
  const bool vec4 = (n & 3) == 0 && (reinterpret_cast<uintptr_t>(D) & 15) == 0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ag = tid >> 3, pg = tid & 7;  // atom group (32), patch group (8)
  const bool timer = (blockIdx.x == 0 && tid == 0 && stats != nullptr);
  __shared__ unsigned long long s_ph[4];  // phase times (slots 8..11), flushed at the end
  if (timer)
    for (int k = 0; k < 4; ++k) s_ph[k] = 0ull;
  unsigned long long tmark = timer ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timer) {
      const unsigned long long t = globaltimer_ns();
      s_ph[slot - 8] += t - tmark;
      tmark = t;
    }
  };

  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t p0 = tile * kSP;
    const int np = (N - p0 < kSP) ? int(N - p0) : kSP;
    const float* Yt = Y + p0 * n;
    for (int t = tid; t < kSP * n; t += kSThreads) {
      const int p = t / n, k = t - p * n;
      const float v = (p < np) ? __ldg(Yt + t) : 0.0f;
      Ys[p * ysn + k] = v;
      Rk[k * rks + p] = v;
    }
    if (tid < kSP) {
      cnt[tid] = 0;
      done[tid] = (tid >= np);
    }
    __syncthreads();
    lap(10);

    for (int step = 0; step < L; ++step) {
      const int live0 = (tid < kSP) ? !done[tid] : 0;
      if (!__syncthreads_or(live0)) break;
      npart[warp * kSP + lane] = 0.0f;

      // ---- residual rows and correlation, chunk by chunk --------------------
      float acc[APT][4];
#pragma unroll
      for (int i = 0; i < APT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
      for (int k0 = 0; k0 < n; k0 += KC) {
        const int kc = min(KC, n - k0);
        __syncthreads();  // the previous chunk is no longer read
        if (vec4) {  // 16-byte loads along each atom row, several in flight
          constexpr int kB = 8;
          const int kc4 = kc >> 2, tot = Kpad * kc4;
          for (int f0 = tid; f0 < tot; f0 += kSThreads * kB) {
            float4 v[kB];
#pragma unroll
            for (int u = 0; u < kB; ++u) {
              const int f = f0 + u * kSThreads;
              const int a = f / kc4, k4 = f - a * kc4;
              v[u] = (f < tot && a < K) ? __ldg(reinterpret_cast<const float4*>(D + int64_t(a) * n + k0) + k4)
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kB; ++u) {
              const int f = f0 + u * kSThreads;
              if (f < tot) {
                const int a = f / kc4, k = 4 * (f - a * kc4);
                Dk[k * dks + a] = v[u].x;
                Dk[(k + 1) * dks + a] = v[u].y;
                Dk[(k + 2) * dks + a] = v[u].z;
                Dk[(k + 3) * dks + a] = v[u].w;
              }
            }
          }
        } else {
          constexpr int kB = 8;
          const int tot = Kpad * kc;
          for (int f0 = tid; f0 < tot; f0 += kSThreads * kB) {
            float v[kB];
#pragma unroll
            for (int u = 0; u < kB; ++u) {
              const int f = f0 + u * kSThreads;
              const int a = f / kc, k = f - a * kc;
              v[u] = (f < tot && a < K) ? __ldg(D + int64_t(a) * n + k0 + k) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kB; ++u) {
              const int f = f0 + u * kSThreads;
              if (f < tot) {
                const int a = f / kc, k = f - a * kc;
                Dk[k * dks + a] = v[u];
              }
            }
          }
        }
        __syncthreads();
        if (step > 0) {  // r = y - D_S g on rows [k0, k0 + kc): lanes over patches
          const int p = lane;
          float nrm = 0.0f;
          if (!done[p]) {
            const int kk = cnt[p];
            for (int k = warp; k < kc; k += kSThreads / 32) {
              float r = Ys[p * ysn + k0 + k];
              for (int s2 = 0; s2 < kk; ++s2) r = fmaf(-gam[p * L + s2], Dk[k * dks + S[p * L + s2]], r);
              Rk[(k0 + k) * rks + p] = r;
              nrm = fmaf(r, r, nrm);
            }
          }
          npart[warp * kSP + p] += nrm;
          __syncthreads();
        }
        const float* dcol = Dk + ag * APT;
        const float* rcol = Rk + pg * 4;
#pragma unroll 2
        for (int k = 0; k < kc; ++k) {
          float dv[APT];
#pragma unroll
          for (int i4 = 0; i4 < APT / 4; ++i4) {
            const float4 d4 = *reinterpret_cast<const float4*>(dcol + k * dks + 4 * i4);
            dv[4 * i4] = d4.x;
            dv[4 * i4 + 1] = d4.y;
            dv[4 * i4 + 2] = d4.z;
            dv[4 * i4 + 3] = d4.w;
          }
          const float4 r = *reinterpret_cast<const float4*>(rcol + (k0 + k) * rks);
          const float rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
          for (int i = 0; i < APT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(dv[i], rv[j], acc[i][j]);
        }
      }
      // ---- residual norms: stop below 1e-3 ----------------------------------
      __syncthreads();
      if (step > 0 && tid < kSP && !done[tid]) {
        float nrm = 0.0f;
        for (int w = 0; w < 8; ++w) nrm += npart[w * kSP + tid];
        if (sqrtf(nrm) < 1e-3f) done[tid] = 1;
      }
      // ---- argmax per patch --------------------------------------------------
      float bv[4];
      int bi[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bv[j] = -1.0f;
        bi[j] = 0x7fffffff;
      }
#pragma unroll
      for (int i = 0; i < APT; ++i) {
        const int a = ag * APT + i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float v = fabsf(acc[i][j]);
          if (a < K && v > bv[j]) {
            bv[j] = v;
            bi[j] = a;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int off = 8; off <= 16; off <<= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, bv[j], off);
          const int oi = __shfl_xor_sync(0xffffffffu, bi[j], off);
          if (s_better(ov, oi, bv[j], bi[j])) {
            bv[j] = ov;
            bi[j] = oi;
          }
        }
      }
      if (lane < 8) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          redv[warp * kSP + pg * 4 + j] = bv[j];
          redi[warp * kSP + pg * 4 + j] = bi[j];
        }
      }
      __syncthreads();
      if (tid < kSP) {
        float v = redv[tid];
        int i = redi[tid];
        for (int w = 1; w < 8; ++w) {
          const float ov = redv[w * kSP + tid];
          const int oi = redi[w * kSP + tid];
          if (s_better(ov, oi, v, i)) {
            v = ov;
            i = oi;
          }
        }
        sel[tid] = (i < K) ? i : 0;
      }
      __syncthreads();
      lap(8);
      const int live = (tid < kSP) ? !done[tid] : 0;
      if (!__syncthreads_or(live)) break;

      // ---- least squares on the grown support -------------------------------
      // (1) dependence test and support-Gram column
      for (int t = tid; t < kSP * (L + 1); t += kSThreads) {
        const int p = t / (L + 1), i = t - p * (L + 1);
        if (done[p]) continue;
        const int k = cnt[p], a = sel[p];
        if (i < k) {
          const int si = S[p * L + i];
          if (si == a) done[p] = 2;  // re-selected atom: the pursuit of p ends
          gS[p * (L + 1) + i] = Gram[int64_t(si) * K + a];
        } else if (i == k) {
          gS[p * (L + 1) + i] = Gram[int64_t(a) * K + a];
        }
      }
      // (2) b_p = d_a . y_p in FP64, four patches per warp
      for (int q = 0; q < kSP / 8; ++q) {
        const int p = warp * (kSP / 8) + q;
        const int a = sel[p];
        double bp = 0.0;
        for (int k = lane; k < n; k += 32) bp = fma(double(__ldg(D + int64_t(a) * n + k)), double(Ys[p * ysn + k]), bp);
        bp = warp_sum(bp);
        if (lane == 0) bS[p] = bp;
      }
      __syncthreads();
      // (3) Cholesky row append and solve, one thread per patch
      if (tid < kSP) {
        const int p = tid;
        if (done[p] == 2) done[p] = 1;
        if (!done[p]) {
          const int k = cnt[p], a = sel[p];
          double* Lp = Lc + p * L * L;
          const double* g = gS + p * (L + 1);
          double ww = 0.0;
          for (int i = 0; i < k; ++i) {
            double s = g[i];
            for (int j2 = 0; j2 < i; ++j2) s -= Lp[i * L + j2] * Lp[k * L + j2];
            const double wi = s * Lp[i * L + i];  // the diagonal is kept as 1 / L_ii
            Lp[k * L + i] = wi;
            ww += wi * wi;
          }
          const double piv2 = g[k] - ww;
          if (!(piv2 > 0.0)) {
            done[p] = 1;  // the new atom depends linearly on the support
          } else {
            const double il = 1.0 / sqrt(piv2);
            Lp[k * L + k] = il;
            S[p * L + k] = a;
            // bvec holds the forward solution z = L^-1 b of the support so
            // far; only its new element is computed
            double zk = bS[p];
            for (int j2 = 0; j2 < k; ++j2) zk -= Lp[k * L + j2] * bvec[p * L + j2];
            bvec[p * L + k] = zk * il;
            cnt[p] = k + 1;
            double yv[kSLMax];
            for (int i = k; i >= 0; --i) {
              double s = bvec[p * L + i];
              for (int j2 = i + 1; j2 <= k; ++j2) s -= Lp[j2 * L + i] * yv[j2];
              yv[i] = s * Lp[i * L + i];
            }
            for (int i = 0; i <= k; ++i) gam[p * L + i] = float(yv[i]);
          }
        }
      }
      __syncthreads();
      lap(9);
    }

    // ---- compact codes ------------------------------------------------------
    for (int t = tid; t < np * L; t += kSThreads) {
      const int p = t / L, s = t - p * L;
      const bool used = s < cnt[p];
      idx_out[(p0 + p) * L + s] = used ? S[p * L + s] : -1;
      coef_out[(p0 + p) * L + s] = used ? gam[p * L + s] : 0.0f;
    }
    __syncthreads();
    lap(10);
  }
  if (timer)
    for (int k = 0; k < 4; ++k) atomicAdd(&stats->phase_ns[8 + k], s_ph[k]);
}

static int s_apt(int K) {
  if (K <= 128) return 4;
  if (K <= 256) return 8;
  if (K <= 512) return 16;
  if (K <= 1024) return 32;
  return 0;
}

static void* s_fn(int apt) {
  switch (apt) {
    case 4: return reinterpret_cast<void*>(omp_stream_kernel<4>);
    case 8: return reinterpret_cast<void*>(omp_stream_kernel<8>);
    case 16: return reinterpret_cast<void*>(omp_stream_kernel<16>);
    case 32: return reinterpret_cast<void*>(omp_stream_kernel<32>);
    default: return nullptr;
  }
}

bool omp_stream_supported(int n, int K, int L) {
  const int apt = s_apt(K);
  if (apt == 0 || L < 1 || L > kSLMax || n < 1) return false;
  return omp_s_layout(n, apt, L).KC >= 4;
}

cudaError_t launch_omp_stream(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                              int L, int32_t* idx, float* coef, int num_sms, DevStats* stats, cudaStream_t s) {
  const int apt = s_apt(K);
  void* fn = s_fn(apt);
  if (!fn || !omp_stream_supported(n, K, L)) return cudaErrorInvalidValue;
  const size_t smem = omp_s_layout(n, apt, L).total;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int64_t ntiles = (N + kSP - 1) / kSP;
  int grid = int(std::min<int64_t>(ntiles, num_sms));
  void* args[] = {(void*)&patches, (void*)&N,   (void*)&n,    (void*)&dict,   (void*)&gram, (void*)&K,
                  (void*)&L,       (void*)&idx, (void*)&coef, (void*)&ntiles, (void*)&stats};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kSThreads), args, smem, s);
}

}  // namespace ksvd
